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
