"""Error against the FP64 oracle on every stated configuration, at full length.

The north star states ψ, E and μ error of the complex64 path against a
complex128 FP64 run at the same dt for every configuration.  These tests run
the configurations at their stated sizes and lengths and check:

* config 2 (stirring, 128^3, box [-12,12)^3, g = 1000, dt = 5e-4, 5000 steps
  from the FP64 ground state): complex64 against the complex128 plan;
* config 3 (large single solve, 256^3, g = 2000, dt = 2.5e-4, 2000 steps with
  n(k) every 100 steps, in 256 uniform bins and in the reference's shell
  binning): complex64 against complex128; the 512^3 leg for 100 steps;
* the complex128 GPU run itself against the CPU oracle (``oracle/ssf.py``,
  scipy.fft in FP64) at 256^3 for 10 stirred steps, so the complex128 plan the
  large configurations are compared with is pinned at full size as well (the
  reference-run fixtures pin it up to 64^3).

Oscillator units (``exp(-i dt k^2/2)``, ``V = ½(x² + 1.44y² + 2.25z²)``) map
exactly onto the reference's convention: ``V_ref = 2V``, ``beta = 2g``,
``dt_ref = dt/2``.  The stirring beam (A = 10, w = 0.5, R = 2, rate ramped
0 -> 0.5 over 200 steps) is mapped the same way.

Gates: ψ ≤ 1e-5 after 1000 steps (north star), ≤ 1e-4 at any point (the
north star's overall bound); N conserved to 1e-6; E and μ within 1e-7 on the
relaxed state and after the first 100 steps, within 1.5e-6 after that; n(k)
per-shell occupation within 1e-5 relative L2 and identical shell counts.

Why E and μ are held to 1.5e-6 on long stirred runs: complex64 storage rounds
the few dominant modes of the condensate every sweep, so the complex64 norm
performs a random walk (about 1e-7 per few hundred steps, either sign; measured
4e-7 after 1300-3000 steps at 128^3 and 256^3) while the complex128 norm stays
within 1e-12.  E follows N with a factor of about 1.4 (E_kin and E_pot scale
with N, E_int with N^2), μ with about 0.5, and E/N stays within 1e-7.

With ``GPE_ACCURACY_OUT`` set, every checkpoint is appended there as a JSON
line (the source of the error table in the design notes).
"""

import json
import os

import numpy as np
import pytest
import torch

from oracle import ssf

pytestmark = pytest.mark.gpu

TRAP = "x**2+1.44*y**2+2.25*z**2"     # 2 x ½(x² + 1.44y² + 2.25z²): reference units


def record(**row):
    path = os.environ.get("GPE_ACCURACY_OUT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(row) + "\n")


def rel_err(a, b):
    """Relative L2 of a against b, on the device, in FP64."""
    d = a.to(torch.complex128) - b.to(torch.complex128)
    return float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b.to(torch.complex128)))


def ground_state(n, L, g, seed=0, dt=1e-3, max_steps=5000, tol=1e-9):
    """FP64 imaginary-time ground state of the trap (reference units), run until
    the energy changes by less than ``tol`` relative per step, or ``max_steps``."""
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, L)
    imag = Plan(n, x, k, dtype=torch.complex128, kind="imaginary", beta=2 * g, dt=dt / 2, static_expr=TRAP)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=seed)).cuda()
    chunk, done, e_prev = 20, 0, None
    while done < max_steps:
        imag.step(psi, chunk, done)
        done += chunk
        e = imag.diagnostics(psi)["E"]
        if e_prev is not None and abs(e - e_prev) / abs(e) < tol * chunk:
            break
        e_prev = e
    imag.close()
    return psi, done


def stir_plans(n, L, g, dt, nk_bins=0, dtypes=(torch.complex64, torch.complex128)):
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    x, k = ssf.get_grids(n, L)
    beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * dt)
    return [Plan(n, x, k, dtype=d, kind="real", beta=2 * g, dt=dt / 2, static_expr=TRAP, beam=beam,
                 nk_bins=nk_bins) for d in dtypes]


def compare(tag, step, p64, p128, a, b, t, nk=False):
    d64, d128 = p64.diagnostics(a, t=t, nk=nk), p128.diagnostics(b, t=t, nk=nk)
    row = dict(config=tag, step=step, psi=rel_err(a, b),
               N=abs(d64["N"] - d128["N"]) / d128["N"],
               E=abs(d64["E"] - d128["E"]) / abs(d128["E"]),
               mu=abs(d64["mu"] - d128["mu"]) / abs(d128["mu"]),
               E_kin=abs(d64["E_kin"] - d128["E_kin"]) / abs(d128["E_kin"]))
    if nk:
        assert np.array_equal(d64["counts"], d128["counts"])
        row["nk"] = float(np.linalg.norm(d64["Nk"] - d128["Nk"]) / np.linalg.norm(d128["Nk"]))
    record(**row)
    return row, d64, d128


def reference_binning_error(a, b, n, L):
    """n(k) in the reference's shells (``gpe/nk_extraction.py:16-45``) of both states."""
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.nk_extraction import nk_extraction
    x, k = helper.get_grids(n, L)
    r64 = nk_extraction(helper.fftn(a, x), x, k)
    r128 = nk_extraction(helper.fftn(b, x), x, k)
    assert np.array_equal(r64["counts"], r128["counts"])
    return float(np.linalg.norm(r64["Nk"] - r128["Nk"]) / np.linalg.norm(r128["Nk"]))


def test_config2_stirring_128_full_5000_steps(cuda):
    n, L, g, dt = 128, 24.0, 1000.0, 5e-4
    psi0, relax = ground_state(n, L, g)
    p64, p128 = stir_plans(n, L, g, dt)
    a = psi0.to(torch.complex64).contiguous()
    b = psi0.clone()
    row, _, _ = compare("2:128", 0, p64, p128, a, b, 0.0)
    for key in ("N", "E", "mu"):
        assert row[key] < 1e-7, row
    n0 = p64.norm(a)
    worst = {}
    for s0 in range(0, 5000, 1000):
        p64.step(a, 1000, s0)
        p128.step(b, 1000, s0)
        row, _, _ = compare("2:128", s0 + 1000, p64, p128, a, b, (s0 + 1000) * dt / 2)
        for key, v in row.items():
            if isinstance(v, float):
                worst[key] = max(worst.get(key, 0.0), v)
        if s0 == 0:
            assert row["psi"] < 1e-5, row
        assert row["psi"] < 1e-4, row
        assert row["N"] < 1e-6, row
        assert row["E"] < 1.5e-6 and row["mu"] < 1.5e-6, row
    drift = abs(p64.norm(a) - n0) / n0
    record(config="2:128", summary=True, relax_steps=relax, norm_drift_c64=drift, **worst)
    assert drift < 1e-6, drift


def test_config3_large_256_full_2000_steps(cuda):
    n, L, g, dt = 256, 24.0, 2000.0, 2.5e-4
    psi0, relax = ground_state(n, L, g, max_steps=3000)
    p64, p128 = stir_plans(n, L, g, dt, nk_bins=256)
    a = psi0.to(torch.complex64).contiguous()
    b = psi0
    worst = {}
    for s0 in range(0, 2000, 100):
        p64.step(a, 100, s0)
        p128.step(b, 100, s0)
        step = s0 + 100
        row, _, _ = compare("3:256", step, p64, p128, a, b, step * dt / 2, nk=True)
        for key, v in row.items():
            if isinstance(v, float):
                worst[key] = max(worst.get(key, 0.0), v)
        if step <= 1000:
            assert row["psi"] < 1e-5, row
        assert row["psi"] < 1e-4, row
        assert row["N"] < 1e-6, row
        tol = 1e-7 if step <= 100 else 1.5e-6
        assert row["E"] < tol and row["mu"] < tol, row
        assert row["nk"] < 1e-5, row
        if step in (1000, 2000):
            ref_nk = reference_binning_error(a, b, n, L)
            record(config="3:256", step=step, nk_reference_binning=ref_nk)
            assert ref_nk < 1e-5, ref_nk
    record(config="3:256", summary=True, relax_steps=relax, **worst)


def test_config3_large_512_against_complex128(cuda):
    """512^3: the register-resident complex64 sweeps against the complex128 plan
    (generic sweeps) for 100 steps from the relaxed 256^3 state's recipe at 512^3
    (a shorter relaxation: 200 imaginary-time steps)."""
    n, L, g, dt = 512, 24.0, 2000.0, 2.5e-4
    psi0, relax = ground_state(n, L, g, max_steps=200)
    p64, p128 = stir_plans(n, L, g, dt, nk_bins=256)
    a = psi0.to(torch.complex64).contiguous()
    b = psi0
    for s0 in (0, 50):
        p64.step(a, 50, s0)
        p128.step(b, 50, s0)
        row, _, _ = compare("3:512", s0 + 50, p64, p128, a, b, (s0 + 50) * dt / 2, nk=True)
        assert row["psi"] < 1e-5, row
        assert row["N"] < 1e-6, row
        assert row["E"] < 1.5e-6 and row["mu"] < 1.5e-6, row
        assert row["nk"] < 1e-5, row
    record(config="3:512", summary=True, relax_steps=relax)


def test_complex128_gpu_matches_cpu_oracle_at_256(cuda):
    """The complex128 plan against the FP64 CPU oracle at 256^3: 10 stirred steps
    (beam during its ramp, g = 2000) from a seeded noisy Gaussian."""
    n, L, g, dt = 256, 24.0, 2000.0, 2.5e-4
    x, _ = ssf.get_grids(n, L)
    psi0 = ssf.noisy_gaussian(x, seed=7)
    (p128,) = stir_plans(n, L, g, dt, dtypes=(torch.complex128,))
    b = torch.from_numpy(psi0).cuda()
    p128.step(b, 10, 0)
    beam = ssf.Beam(2 * 10.0, 0.5, 2.0, 2 * 0.5, 0.5 * 200 * dt)
    m = ssf.Model(n=n, simulation_range=L, kind="real", beta=2 * g, dt=dt / 2, static_expr=TRAP, beam=beam)
    want = ssf.run(psi0, m, 10)
    err = ssf.rel_l2(b.cpu().numpy(), want)
    e_gpu = p128.diagnostics(b, t=10 * dt / 2)
    e_cpu = ssf.energies(want, m, t=10 * dt / 2)
    dE = abs(e_gpu["E"] - e_cpu["E"]) / abs(e_cpu["E"])
    dmu = abs(e_gpu["mu"] - e_cpu["mu"]) / abs(e_cpu["mu"])
    record(config="c128-vs-cpu:256", step=10, psi=err, E=dE, mu=dmu)
    assert err < 1e-12, err
    assert dE < 1e-12 and dmu < 1e-12, (dE, dmu)
