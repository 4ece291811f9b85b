"""The renormalisation entry point that allocates no device memory.

``gpe_normalise_noalloc`` exists for callers that cannot call cudaMalloc: host
frameworks whose memory pool already holds the free HBM, and plugin hosts that
forbid allocation inside their step callbacks.  Its reduction scratch is a
file-scope device array shared by every call on a GPU.  This file runs last
(``test_zz_``) so that a ``-x`` run has already run every other test if it
fails; it passes alone in a fresh process as well.

Checked through the C ABI against the plan-based entry points (``gpe_norm`` +
``gpe_normalise``) on two consecutive calls, for both precisions.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def lib():
    from gpe_simulator_b200 import _lib, build
    build.build()
    return _lib.load(), _lib


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def existing(psi, n, L):
    """Norm and normalised copy through the plan-based entry points."""
    from gpe_simulator_b200 import Plan
    x = np.linspace(-L / 2, L / 2, n, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(n, L / n)
    plan = Plan(n, x, k, dtype=psi.dtype, kind="imaginary", beta=0.0, dt=0.0)
    out = psi.clone()
    N = plan.norm(out)
    plan.normalise(out)
    torch.cuda.synchronize()
    plan.close()
    return N, out, x[1] - x[0]


@pytest.mark.parametrize("dtype,code,tol", [(torch.complex128, 1, 1e-13), (torch.complex64, 0, 1e-6)])
def test_two_calls_match_plan_based_normalise(cuda, dtype, code, tol):
    so, _lib = lib()
    g = torch.Generator(device="cuda").manual_seed(11)
    for n, L in ((48, 9.0), (64, 12.0)):  # two calls in a row, different grids
        psi = (torch.randn((n, n, n), dtype=dtype, device="cuda", generator=g) * 3.0).contiguous()
        want_N, want, dx = existing(psi, n, L)
        got = psi.clone()
        N = ctypes.c_double()
        rc = so.gpe_normalise_noalloc(ctypes.c_void_p(got.data_ptr()), n, code, dx, ctypes.byref(N), stream())
        assert rc == _lib.GPE_OK, _lib.last_error()
        assert N.value == pytest.approx(want_N, rel=1e-13)
        err = ((got - want).abs().pow(2).sum() / want.abs().pow(2).sum()).sqrt().item()
        assert err < tol, err
        # the result is normalised: a second call finds N = 1 and leaves psi unchanged
        again = got.clone()
        rc = so.gpe_normalise_noalloc(ctypes.c_void_p(again.data_ptr()), n, code, dx, ctypes.byref(N), stream())
        assert rc == _lib.GPE_OK, _lib.last_error()
        assert N.value == pytest.approx(1.0, abs=10 * tol)
        err = ((again - got).abs().pow(2).sum() / got.abs().pow(2).sum()).sqrt().item()
        assert err < tol, err


def test_no_device_memory_is_allocated(cuda):
    """After the first call in the context (which also loads both precisions'
    kernels), calls of either precision take no device memory."""
    so, _lib = lib()
    n = 32
    psi64 = torch.ones((n, n, n), dtype=torch.complex64, device="cuda")
    psi128 = torch.ones((n, n, n), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    # first call: set-up in this context
    assert so.gpe_normalise_noalloc(ctypes.c_void_p(psi64.data_ptr()), n, 0, 0.5, None, stream()) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert so.gpe_normalise_noalloc(ctypes.c_void_p(psi128.data_ptr()), n, 1, 0.5, None, stream()) == 0
        assert so.gpe_normalise_noalloc(ctypes.c_void_p(psi64.data_ptr()), n, 0, 0.5, None, stream()) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    dx3 = 0.5 ** 3
    assert float(psi64.abs().pow(2).sum()) * dx3 == pytest.approx(1.0, rel=1e-5)
    assert float(psi128.abs().pow(2).sum()) * dx3 == pytest.approx(1.0, rel=1e-13)


@pytest.mark.parametrize("dtype,code", [(torch.complex64, 0), (torch.complex128, 1)])
def test_zero_or_nonfinite_norm_is_reported_and_psi_left_unchanged(cuda, dtype, code):
    """The plan path flags a zero norm through its status word; this entry point
    returns GPE_ERR_NONFINITE and leaves psi as it was (no division by zero)."""
    so, _lib = lib()
    n = 16
    for fill in (0.0, float("nan")):
        psi = torch.full((n, n, n), fill, dtype=dtype, device="cuda")
        before = psi.clone()
        N = ctypes.c_double(-1.0)
        rc = so.gpe_normalise_noalloc(ctypes.c_void_p(psi.data_ptr()), n, code, 0.25, ctypes.byref(N), stream())
        assert rc == _lib.GPE_ERR_NONFINITE, rc
        assert "norm" in _lib.last_error()
        assert torch.equal(psi.isnan(), before.isnan())
        assert torch.equal(torch.nan_to_num(psi), torch.nan_to_num(before))
        # the same status without a norm pointer
        rc = so.gpe_normalise_noalloc(ctypes.c_void_p(psi.data_ptr()), n, code, 0.25, None, stream())
        assert rc == _lib.GPE_ERR_NONFINITE
    # a finite state afterwards is normalised again (the status word was cleared)
    psi = torch.ones((n, n, n), dtype=dtype, device="cuda")
    assert so.gpe_normalise_noalloc(ctypes.c_void_p(psi.data_ptr()), n, code, 0.25, None, stream()) == 0
    assert float(psi.abs().pow(2).sum()) * 0.25 ** 3 == pytest.approx(1.0, rel=1e-5)


def test_rejects_sizes_beyond_the_maximum(cuda):
    so, _lib = lib()
    psi = torch.ones(8, dtype=torch.complex64, device="cuda")
    rc = so.gpe_normalise_noalloc(ctypes.c_void_p(psi.data_ptr()), 1025, 0, 0.1, None, stream())
    assert rc == _lib.GPE_ERR_UNSUPPORTED
    assert "1024" in _lib.last_error()
    rc = so.gpe_normalise_noalloc(ctypes.c_void_p(psi.data_ptr()), 2, 5, 0.1, None, stream())
    assert rc == _lib.GPE_ERR_ARG
