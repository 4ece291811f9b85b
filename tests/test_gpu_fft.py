"""3-D FFT of the fused sweeps vs numpy.fft (``cp.fft.fftn`` / ``ifftn`` contract)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SIZES = [2, 4, 7, 8, 12, 16, 18, 30, 32, 48, 64, 96, 128, 160]


def _plan(n, dtype):
    from gpe_simulator_b200 import Plan
    from oracle.ssf import get_grids
    x, k = get_grids(n, 10.0)
    return Plan(n, x, k, dtype=dtype, kind="imaginary", beta=0.0, dt=0.0)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-13), (torch.complex64, 2e-6)])
def test_forward_inverse_match_numpy(cuda, n, dtype, tol):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    plan = _plan(n, dtype)
    src = torch.from_numpy(a).to(dtype).cuda()
    ref = np.fft.fftn(src.cpu().numpy().astype(np.complex128))
    out = plan.fft(src)
    err = np.linalg.norm(out.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < tol, err
    back = plan.fft(out, inverse=True)
    err = np.linalg.norm(back.cpu().numpy() - src.cpu().numpy()) / np.linalg.norm(a)
    assert err < tol, err
    # input untouched by the out-of-place transform
    assert torch.equal(src, torch.from_numpy(a).to(dtype).cuda())


def test_in_place_transform(cuda):
    n = 32
    rng = np.random.default_rng(1)
    a = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    plan = _plan(n, torch.complex128)
    t = torch.from_numpy(a).cuda()
    plan.fft(t, out=t)
    np.testing.assert_allclose(t.cpu().numpy(), np.fft.fftn(a), rtol=1e-12, atol=1e-10)


def test_large_grid_roundtrip(cuda):
    n = 256
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.randn((n, n, n), dtype=torch.complex64, device="cuda", generator=g)
    plan = _plan(n, torch.complex64)
    f = plan.fft(a)
    # spot check of a few modes against a direct sum along one line of the cube
    ref = torch.fft.fftn(a.to(torch.complex128))
    err = ((f.to(torch.complex128) - ref).abs().pow(2).sum() / ref.abs().pow(2).sum()).sqrt().item()
    assert err < 2e-6, err
    b = plan.fft(f, inverse=True)
    err = ((b - a).abs().pow(2).sum() / a.abs().pow(2).sum()).sqrt().item()
    assert err < 2e-6, err
