"""The largest grid (n = 1024, generic sweeps, complex64: 8 GiB per cube),
checked through size-independent properties: a plane-wave known answer, the FFT
round trip and Parseval."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N, L = 1024, 40.0


def test_max_grid_plane_wave_and_fft_roundtrip(cuda):
    from gpe_simulator_b200 import Plan
    x = np.linspace(-L / 2, L / 2, N, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(N, L / N)
    dt = 1e-3
    plan = Plan(N, x, k, dtype=torch.complex64, kind="real", beta=0.0, dt=dt)
    # plane wave along y: without potential or interaction one step multiplies it by exp(-i k0^2 dt)
    k0 = float(k[3])
    y = torch.from_numpy(x).cuda()
    wave = torch.exp(1j * k0 * y).to(torch.complex64)
    psi = wave[None, :, None].expand(N, N, N).contiguous()
    plan.normalise(psi)
    amp = psi[0, 0, 0].abs().item()
    plan.step(psi, 2, 0)
    want = (wave * amp * complex(math.cos(2 * k0 ** 2 * dt), -math.sin(2 * k0 ** 2 * dt)))[None, :, None]
    err = ((psi - want).abs().max() / amp).item()
    assert err < 1e-5, err
    assert plan.norm(psi) == pytest.approx(1.0, abs=1e-6)
    del psi, want
    torch.cuda.empty_cache()
    # FFT round trip and Parseval on random data
    g = torch.Generator(device="cuda").manual_seed(11)
    a = torch.randn((N, N, N), dtype=torch.complex64, device="cuda", generator=g)
    f = plan.fft(a)
    pa = a.abs().pow(2).sum(dtype=torch.float64).item()
    pf = f.abs().pow(2).sum(dtype=torch.float64).item()
    assert pf / (N ** 3 * pa) == pytest.approx(1.0, rel=1e-6)
    back = plan.fft(f, inverse=True)
    del f
    err = ((back - a).abs().pow(2).sum(dtype=torch.float64) / pa).sqrt().item()
    assert err < 3e-6, err


@pytest.mark.parametrize("path", ["per_step", "multi_step"])
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-11), (torch.complex64, 2e-5)])
def test_stirred_256_is_time_reversible(cuda, dtype, tol, path):
    """The bench workload (256^3, trap, g = 2000, rotating beam) run forward 50
    real-time steps and back with -dt at the same mid-step times returns to its
    start: Strang splitting with an exact (|psi|-preserving) local step is
    symmetric, so only rounding remains."""
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    from oracle import ssf
    n, L, dt = 256, 24.0, 1.25e-4
    x, k = ssf.get_grids(n, L)
    beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * 2.5e-4)
    kw = dict(dtype=dtype, kind="real", beta=4000.0, static_expr="x**2+1.44*y**2+2.25*z**2", beam=beam)
    fwd, back = Plan(n, x, k, dt=dt, **kw), Plan(n, x, k, dt=-dt, **kw)
    psi0 = torch.from_numpy(ssf.noisy_gaussian(x, seed=9)).to(dtype).cuda()
    fwd.normalise(psi0)
    psi = psi0.clone()
    steps = 50
    if path == "per_step":
        for i in range(steps):
            fwd.step_at(psi, i * dt)             # mid-step time i dt + dt/2
    else:
        fwd.step(psi, steps, 0)                  # one call, fused z sweeps between steps
    moved = ((psi - psi0).abs().pow(2).sum() / psi0.abs().pow(2).sum()).sqrt().item()
    if path == "per_step":
        for i in reversed(range(steps)):
            back.step_at(psi, i * dt + dt)       # same mid-step time with -dt
    else:
        back.step(psi, steps, -steps)            # step j at (-steps + j)(-dt) - dt/2: the same times reversed
    err = ((psi - psi0).abs().pow(2).sum() / psi0.abs().pow(2).sum()).sqrt().item()
    assert moved > 1e-2                          # the state did evolve
    assert err < tol, err


def test_stirred_512_is_time_reversible(cuda):
    """The 512^3 register-resident sweeps (complex64): 20 fused steps forward and
    20 back with -dt return to the start."""
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    n, L, dt = 512, 24.0, 1.25e-4
    x = np.linspace(-L / 2, L / 2, n, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(n, L / n)
    beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * 2.5e-4)
    kw = dict(dtype=torch.complex64, kind="real", beta=4000.0, static_expr="x**2+1.44*y**2+2.25*z**2",
              beam=beam)
    fwd, back = Plan(n, x, k, dt=dt, **kw), Plan(n, x, k, dt=-dt, **kw)
    g = torch.from_numpy(np.exp(-x ** 2 / 2)).cuda()
    psi0 = (g[:, None, None] * g[None, :, None] * g[None, None, :]).to(torch.complex64)
    psi0 = psi0 * (1 + 0.01 * torch.randn(psi0.shape, dtype=torch.complex64, device="cuda",
                                          generator=torch.Generator(device="cuda").manual_seed(3)))
    fwd.normalise(psi0)
    psi = psi0.clone()
    fwd.step(psi, 20, 0)
    moved = ((psi - psi0).abs().pow(2).sum() / psi0.abs().pow(2).sum()).sqrt().item()
    back.step(psi, 20, -20)
    err = ((psi - psi0).abs().pow(2).sum() / psi0.abs().pow(2).sum()).sqrt().item()
    assert moved > 1e-3
    assert err < 2e-5, err
