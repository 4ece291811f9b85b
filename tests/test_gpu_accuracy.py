"""complex64 accuracy gates of the real-time stirring workload (128^3, box
[-12,12)^3, g = 1000, dt = 5e-4 in oscillator units, rotating beam A = 10,
w = 0.5, R = 2, rate ramped 0 -> 0.5 over 200 steps), run in reference units:

* psi after 1000 real-time steps within 1e-5 (relative L2) of the complex128
  run of the same plan from the same state;
* the norm conserved to 1e-6 over 5000 real-time steps;
* E and mu within 1e-7 (relative) of the complex128 values for the relaxed
  state, and within 5e-7 once it has been stirred (1000 steps at 128^3, 100-200
  steps of a barely relaxed state at 256^3).  The stirred complex64 energy
  error follows psi's FP32 rounding error, a random walk (psi 2e-6 after 100
  steps, 6.6e-6 after 1000): N wanders by up to 2e-7 and E by about 1.5 times
  that, with either sign (E/N stays within 8e-8); measured 1e-8 to 2.5e-7, with
  and without FP64 evaluation of the local factor, so it is not a bias.
  complex128 matches the reference to 1e-10 (tests/test_gpu_golden.py).
"""

import numpy as np
import pytest
import torch

from oracle import ssf

pytestmark = pytest.mark.gpu

N, L, G, DT = 128, 24.0, 1000.0, 5e-4
TRAP = "x**2+1.44*y**2+2.25*z**2"


def plans(dtype):
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    x, k = ssf.get_grids(N, L)
    beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * DT)
    real = Plan(N, x, k, dtype=dtype, kind="real", beta=2 * G, dt=DT / 2, static_expr=TRAP, beam=beam)
    return real, x, k


@pytest.fixture(scope="module")
def start(cuda):
    """A relaxed trap state (300 imaginary-time steps in complex128)."""
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(N, L)
    imag = Plan(N, x, k, dtype=torch.complex128, kind="imaginary", beta=2 * G, dt=DT, static_expr=TRAP)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=0)).cuda()
    imag.step(psi, 300)
    torch.cuda.synchronize()
    return psi


def test_complex64_matches_complex128_after_1000_steps(start):
    p64, _, _ = plans(torch.complex64)
    p128, _, _ = plans(torch.complex128)
    a = start.to(torch.complex64).contiguous()
    b = a.to(torch.complex128).contiguous()
    d64, d128 = p64.diagnostics(a, t=0.0), p128.diagnostics(b, t=0.0)
    for key in ("N", "E", "mu"):
        assert abs(d64[key] - d128[key]) / abs(d128[key]) < 1e-7, ("relaxed", key, d64[key], d128[key])
    p64.step(a, 1000, 0)
    p128.step(b, 1000, 0)
    err = ssf.rel_l2(a.cpu().numpy().astype(np.complex128), b.cpu().numpy())
    assert err < 1e-5, err
    d64 = p64.diagnostics(a, t=1000 * DT / 2)
    d128 = p128.diagnostics(b, t=1000 * DT / 2)
    assert abs(d64["N"] - d128["N"]) / d128["N"] < 1e-6, (d64["N"], d128["N"])
    for key in ("E", "mu"):
        assert abs(d64[key] - d128[key]) / abs(d128[key]) < 5e-7, ("stirred", key, d64[key], d128[key])


def test_complex64_norm_conserved_over_5000_steps(start):
    p64, _, _ = plans(torch.complex64)
    a = start.to(torch.complex64).contiguous()
    n0 = p64.norm(a)
    for s0 in range(0, 5000, 1000):
        p64.step(a, 1000, s0)
    n1 = p64.norm(a)
    assert abs(n1 - n0) / n0 < 1e-6, (n0, n1)


def test_large_256_against_complex128_with_nk():
    """Large single solve, 256^3 (box [-12,12)^3, g = 2000, dt = 2.5e-4, beam),
    complex64 against the complex128 run from the same state: psi, E, mu and
    n(k) in 256 radial bins after 100 and 200 real-time steps."""
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    n = 256
    x, k = ssf.get_grids(n, 24.0)
    relax = Plan(n, x, k, dtype=torch.complex128, kind="imaginary", beta=4000.0, dt=2.5e-4, static_expr=TRAP)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=3)).cuda()
    relax.step(psi, 50)
    relax.close()
    beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * 2.5e-4)
    p64, p128 = (Plan(n, x, k, dtype=dt_, kind="real", beta=4000.0, dt=1.25e-4, static_expr=TRAP, beam=beam,
                      nk_bins=256) for dt_ in (torch.complex64, torch.complex128))
    a = psi.to(torch.complex64).contiguous()
    b = psi
    for s0 in (0, 100):
        p64.step(a, 100, s0)
        p128.step(b, 100, s0)
        t = (s0 + 100) * 1.25e-4
        d64, d128 = p64.diagnostics(a, t=t, nk=True), p128.diagnostics(b, t=t, nk=True)
        err = ssf.rel_l2(a.cpu().numpy().astype(np.complex128), b.cpu().numpy())
        assert err < 1e-5, (s0, err)
        assert abs(d64["N"] - d128["N"]) / d128["N"] < 1e-7, (s0, d64["N"], d128["N"])
        for key in ("E", "mu"):
            assert abs(d64[key] - d128[key]) / abs(d128[key]) < 5e-7, (s0, key, d64[key], d128[key])
        assert np.array_equal(d64["counts"], d128["counts"])
        nk_err = np.linalg.norm(d64["Nk"] - d128["Nk"]) / np.linalg.norm(d128["Nk"])
        assert nk_err < 1e-5, (s0, nk_err)


def test_stage_run_logs_norm_and_energy_every_50_steps(tmp_path):
    """Real-time stirring at 128^3 through the stage API: 5000 steps with N and E
    logged every 50 steps (launch_stage runs the steps between log points as
    one call); the norm stays within 1e-6 at every log point."""
    from gpe_simulator_b200 import beam_in_reference_units, helper
    from gpe_simulator_b200.expressions import cuda_expression
    from gpe_simulator_b200.launch import launch_stage
    from gpe_simulator_b200.stage import stage
    x, k = helper.get_grids(N, L)
    pp = dict(static=dict(activate=True, expression=cuda_expression(TRAP)),
              dynamic=dict(activate=False, expression="0"))
    st = stage(simulation_range=L, x_array=x, k_array=k, N_grids=N, type="real", steps=5000, dt=DT / 2,
               initial_state=dict(type="continue"), box_params=dict(activate=False),
               absorber_params=dict(activate=False), noise_params=dict(activate=False),
               cloud_params=dict(a=0.0, N_atom=1), monitor_params={},
               save_params=dict(scalar_interval=50, nk_interval=0), potential_params=pp,
               k_cut_params=dict(activate=False, k_cut=0.0), precision="complex64",
               beam=beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * DT))
    st.beta = 2 * G
    start = torch.from_numpy(ssf.noisy_gaussian(x.cpu().numpy(), seed=0)).cuda()
    st.prepare(previous_psi=start)
    st.monitor_dir = tmp_path
    launch_stage(st)
    hist = st.history
    assert [h["step"] for h in hist] == list(range(50, 5001, 50))
    n0 = hist[0]["N"]
    assert max(abs(h["N"] - n0) for h in hist) / n0 < 1e-6
    assert all(np.isfinite(h["E"]) for h in hist)
    rows = (tmp_path / "scalars.csv").read_text().strip().splitlines()
    assert len(rows) == 1 + 100
    assert rows[0].split(",")[:6] == ["step", "time", "norm", "N_atoms", "E_kin", "Lz"]
    assert all(np.isfinite(h["Lz"]) for h in hist)


def test_stage_snapshots_round_trip(tmp_path):
    """launch_stage writes psi snapshots (complex128 files) at psi_interval and at
    the end; a complex64 stage reloads the last one exactly."""
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.expressions import cuda_expression
    from gpe_simulator_b200.launch import launch_stage
    from gpe_simulator_b200.stage import stage

    def make(initial):
        x, k = helper.get_grids(32, 10.0)
        return stage(simulation_range=10.0, x_array=x, k_array=k, N_grids=32, type="imaginary", steps=6,
                     dt=1e-3, initial_state=initial, box_params=dict(activate=False),
                     absorber_params=dict(activate=False), noise_params=dict(activate=False),
                     cloud_params=dict(a=0.0, N_atom=1), monitor_params={},
                     save_params=dict(scalar_interval=0, nk_interval=0, psi_interval=4, save_final=True),
                     potential_params=dict(static=dict(activate=True, expression=cuda_expression("x**2+y**2+z**2")),
                                           dynamic=dict(activate=False, expression="0")),
                     k_cut_params=dict(activate=False, k_cut=0.0), precision="complex64")
    st = make(dict(type="gaussian", sigma=1.0))
    st.prepare()
    st.data_dir = tmp_path
    psi = launch_stage(st)
    assert sorted(f.name for f in tmp_path.glob("psi_*.npy")) == ["psi_00000004.npy", "psi_00000006.npy"]
    st2 = make(dict(type="load", path=str(tmp_path / "psi_00000006.npy")))
    st2.prepare()
    assert st2.psi.dtype == torch.complex64 and torch.equal(st2.psi, psi)
