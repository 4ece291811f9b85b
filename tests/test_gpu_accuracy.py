"""complex64 accuracy gates of the real-time stirring workload (128^3, box
[-12,12)^3, g = 1000, dt = 5e-4 in oscillator units, rotating beam A = 10,
w = 0.5, R = 2, rate ramped 0 -> 0.5 over 200 steps), run in reference units:

* psi after 1000 real-time steps within 1e-5 (relative L2) of the complex128
  run of the same plan from the same state;
* the norm conserved to 1e-6 over 5000 real-time steps;
* E and mu after 1000 steps within 1e-7 (relative) of the complex128 values.
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
    p64.step(a, 1000, 0)
    p128.step(b, 1000, 0)
    err = ssf.rel_l2(a.cpu().numpy().astype(np.complex128), b.cpu().numpy())
    assert err < 1e-5, err
    d64 = p64.diagnostics(a, t=1000 * DT / 2)
    d128 = p128.diagnostics(b, t=1000 * DT / 2)
    assert abs(d64["E"] - d128["E"]) / abs(d128["E"]) < 1e-7, (d64["E"], d128["E"])
    assert abs(d64["mu"] - d128["mu"]) / abs(d128["mu"]) < 1e-7, (d64["mu"], d128["mu"])


def test_complex64_norm_conserved_over_5000_steps(start):
    p64, _, _ = plans(torch.complex64)
    a = start.to(torch.complex64).contiguous()
    n0 = p64.norm(a)
    for s0 in range(0, 5000, 1000):
        p64.step(a, 1000, s0)
    n1 = p64.norm(a)
    assert abs(n1 - n0) / n0 < 1e-6, (n0, n1)
