"""Generate the golden fixtures from the reference implementation itself.

Runs ONLY where the reference sources are present (``GPE_REFERENCE`` or
``/root/reference``).  The reference's own ``gpe`` package is imported with a
NumPy-backed CuPy (``oracle/ref_shim.py``): its propagator closures
(``gpe/make_propagator.py``), its CUDA kernel strings compiled for the host
(``gpe/kernels.py``, ``gpe/make_kernel.py``, ``gpe/helper.py``) and its
diagnostics (``gpe/helper.py:135-140``, ``gpe/nk_extraction.py:16-45``) produce
every number stored here; only cuFFT is replaced by numpy.fft.

All cases are in reference units (kinetic factor ``exp(-i k^2 dt)``).  Inputs
are regenerated from the stored seeds, so the fixtures hold outputs only:

* ``ground64``   config "plain imaginary-time ground state": N=64, box
  [-8,8)^3, V = x^2+1.44y^2+2.25z^2 (= 2 x the oscillator-unit trap),
  beta = 1000 (g = 500), dt = 5e-4 (oscillator dt = 1e-3), seeded noisy
  Gaussian (seed 0), 2000 steps; checkpoints at 100, 1000, 2000.
* ``stir32``     200 imaginary steps from a noisy Gaussian (seed 1), then 400
  real-time steps with the harmonic trap plus a rotating Gaussian beam written
  in the reference's expression grammar.  N=32, box [-12,12)^3, beta = 2000.
* ``lossy16``    real time with a complex static potential (absorber ``-i
  Gamma`` ramp plus a real box) and a momentum cutoff, N=16.
* ``box24``      imaginary time with a float64 box potential array plus a
  static expression, N=24.
* ``diag_n*``    ``get_N``, ``get_E``, ``get_L`` and ``nk_extraction`` of seeded states.

Usage: ``python tests/golden/make_golden.py`` (writes ``tests/golden/*.npz``).
"""

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref_shim, ssf  # noqa: E402
from tests.golden import cases  # noqa: E402

OUT = Path(__file__).resolve().parent


def summary(psi, x, k, ref, sub):
    """Subsampled field, random projections and reference diagnostics of psi."""
    psi = np.ascontiguousarray(psi)
    out = dict(psi_sub=psi[::sub, ::sub, ::sub].copy(),
               proj=cases.projections(psi),
               N=float(ref.helper.get_N(psi, x)),
               E_kin=float(ref.helper.get_E(np.fft.fftn(psi), x, k)))
    return out


def save(name, **arrays):
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print("wrote", name, flush=True)


def make_ground64(ref):
    c = cases.GROUND64
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"])
    psi = ssf.noisy_gaussian(st.x_array, seed=c["seed"])
    out, done = {}, 0
    for mark in c["checkpoints"]:
        t0 = time.time()
        psi = ref_shim.run_reference(ref, st, psi, mark - done, step0=done)
        done = mark
        for key, val in summary(psi, st.x_array, st.k_array, ref, c["sub"]).items():
            out[f"{key}_{mark}"] = val
        print(f"ground64 step {mark} ({time.time() - t0:.0f}s)", flush=True)
    save("ground64", **out)


def make_stir32(ref):
    c = cases.STIR32
    imag = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                    beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"])
    psi = ssf.noisy_gaussian(imag.x_array, seed=c["seed"])
    psi = ref_shim.run_reference(ref, imag, psi, c["imag_steps"])
    start = summary(psi, imag.x_array, imag.k_array, ref, c["sub"])
    real = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="real",
                                    beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                    dynamic_expr=cases.stir_beam().expression())
    out = {"psi_start": start["psi_sub"], "N_start": start["N"]}
    done = 0
    for mark in c["checkpoints"]:
        psi = ref_shim.run_reference(ref, real, psi, mark - done, step0=done)
        done = mark
        for key, val in summary(psi, real.x_array, real.k_array, ref, c["sub"]).items():
            out[f"{key}_{mark}"] = val
    save("stir32", **out)


def make_lossy16(ref):
    c = cases.LOSSY16
    x, _ = ssf.get_grids(c["n"], c["L"])
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="real",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                  dynamic_expr=c["dynamic_expr"], k_cut=c["k_cut"],
                                  static_v=cases.lossy_potential(x, c))
    psi = ssf.noisy_gaussian(x, sigma=1.5, seed=c["seed"])
    psi = ref_shim.run_reference(ref, st, psi, c["steps"])
    save("lossy16", psi=psi, N=float(ref.helper.get_N(psi, st.x_array)))


def make_box24(ref):
    c = cases.BOX24
    x, _ = ssf.get_grids(c["n"], c["L"])
    st = ref_shim.reference_stage(ref, n=c["n"], simulation_range=c["L"], kind="imaginary",
                                  beta=c["beta"], dt=c["dt"], static_expr=c["static_expr"],
                                  static_v=cases.box_potential(x, c))
    psi = ssf.noisy_gaussian(x, sigma=2.0, seed=c["seed"])
    psi = ref_shim.run_reference(ref, st, psi, c["steps"])
    save("box24", psi=psi)


def make_diag(ref):
    for n, L in cases.DIAG_SIZES:
        x, k = ref.grids.get_grids(n, L)
        psi = cases.diag_state(n)
        F = np.fft.fftn(psi)
        spec = ref.nk_extraction.nk_extraction(F, x, k, slab_size=3)
        save(f"diag_n{n}", N=float(ref.helper.get_N(psi, x)),
             E_kin=float(ref.helper.get_E(F, x, k)), L=float(ref.helper.get_L(psi, x, k, slab_size=3)),
             **{f"nk_{key}": np.asarray(val) for key, val in spec.items()})


def main(which=None):
    ref = ref_shim.install()
    jobs = dict(diag=make_diag, lossy16=make_lossy16, box24=make_box24,
                stir32=make_stir32, ground64=make_ground64)
    for name, job in jobs.items():
        if which is None or name in which:
            job(ref)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
