"""Edge cases of the propagator path: the smallest grids and the odd-prime
radices, zero-step calls and states with no norm."""

import numpy as np
import pytest
import torch

from oracle import ssf
from tests.golden import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [2, 3, 5, 13, 26])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_small_and_odd_prime_grids_match_oracle(cuda, n, kind, dtype, tol):
    """Grids of 2 points per axis and the radix-3, 5, 13 (direct) passes: three
    steps against the oracle, the beam included in real time."""
    from gpe_simulator_b200 import Beam, Plan
    x, k = ssf.get_grids(n, 8.0)
    kw = dict(beta=300.0, dt=1e-3, static_expr=cases.TRAP)
    beam = Beam(20.0, 0.8, 1.5, 1.0, 0.002) if kind == "real" else None
    plan = Plan(n, x, k, dtype=dtype, kind=kind, beam=beam, **kw)
    a = torch.from_numpy(ssf.noisy_gaussian(x, sigma=1.5, seed=n)).to(dtype).cuda()
    start = a.cpu().numpy().astype(np.complex128)      # the state as stored (complex64 rounded)
    plan.step(a, 3, 1)
    m = ssf.Model(n=n, simulation_range=8.0, kind=kind, beta=300.0, dt=1e-3, static_expr=cases.TRAP,
                  beam=ssf.Beam(20.0, 0.8, 1.5, 1.0, 0.002) if kind == "real" else None)
    err = ssf.rel_l2(a.cpu().numpy(), ssf.run(start, m, 3, step0=1))
    assert err < tol, err
    assert plan.status() == 0


@pytest.mark.parametrize("n", [22, 26, 39])
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-13), (torch.complex64, 2e-6)])
def test_radix_11_and_13_transforms(cuda, n, dtype, tol):
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, 10.0)
    plan = Plan(n, x, k, dtype=dtype, kind="imaginary", beta=0.0, dt=0.0)
    rng = np.random.default_rng(n)
    a = torch.from_numpy(rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))).to(dtype).cuda()
    ref = np.fft.fftn(a.cpu().numpy().astype(np.complex128))
    f = plan.fft(a)
    assert np.linalg.norm(f.cpu().numpy() - ref) / np.linalg.norm(ref) < tol
    back = plan.fft(f, inverse=True)
    assert ssf.rel_l2(back.cpu().numpy(), a.cpu().numpy()) < tol


@pytest.mark.parametrize("n", [16, 64, 256])
@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_zero_steps_leave_psi_untouched(cuda, n, kind):
    """``nsteps = 0`` launches nothing: no half-step, no renormalisation."""
    from gpe_simulator_b200 import Plan
    from gpe_simulator_b200.plan import launch_count
    x, k = ssf.get_grids(n, 12.0)
    plan = Plan(n, x, k, dtype=torch.complex64, kind=kind, beta=500.0, dt=1e-3, static_expr=cases.TRAP)
    a = 3.0 * torch.from_numpy(ssf.noisy_gaussian(x, seed=2)).to(torch.complex64).cuda()   # not normalised
    b = a.clone()
    n0 = launch_count(plan)
    plan.step(a, 0, 7)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert launch_count(plan) == n0


@pytest.mark.parametrize("n", [32, 48])
def test_state_without_norm_is_flagged(cuda, n):
    """Imaginary time renormalises by 1/sqrt(N): a zero state has no norm, so the
    step raises the non-finite status (bit 0) instead of returning silently; a
    real-time step of the zero state stays zero with a clean status."""
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, 12.0)
    imag = Plan(n, x, k, dtype=torch.complex64, kind="imaginary", beta=500.0, dt=1e-3, static_expr=cases.TRAP)
    real = Plan(n, x, k, dtype=torch.complex64, kind="real", beta=500.0, dt=1e-3, static_expr=cases.TRAP)
    z = torch.zeros((n, n, n), dtype=torch.complex64, device="cuda")
    imag.step(z, 2)
    assert imag.status() & 1
    assert imag.status() == 0          # read and cleared
    w = torch.zeros_like(z)
    real.step(w, 3)
    assert real.status() == 0 and not w.abs().sum().item()
