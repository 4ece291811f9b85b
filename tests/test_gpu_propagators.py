"""The reference's analytic propagator checks, run through the drop-in API.

Restated from the reference's ``tests/test_propagators.py`` (N=8, L=2 pi so k
is an integer; plane waves): real-time phase for all static/dynamic/cutoff
combinations, generated spatial expressions at each grid point (N=7),
imaginary two-mode decay with normalisation, absorber loss and cutoff.
"""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def make_stage(kind, n=8, L=2 * math.pi, a=0.0, static=None, dynamic=None, k_cut=None,
               steps=3, dt=0.01, precision="complex128"):
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.expressions import cuda_expression
    from gpe_simulator_b200.stage import stage
    x, k = helper.get_grids(n, L)
    pp = dict(static=dict(activate=static is not None, expression=cuda_expression(static or "0")),
              dynamic=dict(activate=dynamic is not None,
                           expression=cuda_expression(dynamic or "0", time_dependent=True)))
    st = stage(simulation_range=L, x_array=x, k_array=k, N_grids=n, type=kind, steps=steps, dt=dt,
               initial_state=dict(type="gaussian", sigma=1.0), box_params=dict(activate=False),
               absorber_params=dict(activate=False), noise_params=dict(activate=False),
               cloud_params=dict(a=a, N_atom=150000), monitor_params={},
               save_params=dict(scalar_interval=0, nk_interval=0),
               potential_params=pp,
               k_cut_params=dict(activate=k_cut is not None, k_cut=k_cut or 0.0), precision=precision)
    st.prepare()
    return st


def plane_wave(st, mode=1):
    x = st.x_array.cpu().numpy()
    w = np.exp(1j * mode * x)[:, None, None]
    return np.broadcast_to(w, (st.N_grids,) * 3).copy() / (2 * np.pi) ** 1.5


@pytest.mark.parametrize("precision,rtol,atol", [("complex128", 1e-11, 1e-12), ("complex64", 2e-6, 2e-7)])
def test_real_phase_all_combinations(cuda, precision, rtol, atol):
    from gpe_simulator_b200.helper import get_N
    from gpe_simulator_b200.launch import launch_stage
    for static in (False, True):
        for dynamic in (False, True):
            for cutoff in (False, True):
                st = make_stage("real", a=10, static="1/2" if static else None,
                                dynamic="t/4" if dynamic else None, k_cut=1.5 if cutoff else None,
                                precision=precision)
                init = plane_wave(st)
                st.psi = torch.from_numpy(init).to(st.psi.dtype).cuda()
                T = st.steps * st.dt
                phase = (1 + st.beta / (2 * np.pi) ** 3) * T
                phase += (0.5 * T if static else 0) + (T ** 2 / 8 if dynamic else 0)
                res = launch_stage(st)
                np.testing.assert_allclose(res.cpu().numpy(), init * np.exp(-1j * phase),
                                           rtol=rtol, atol=atol)
                assert abs(get_N(res, st.x_array) - 1) < (1e-11 if precision == "complex128" else 1e-6)


def test_per_step_closures_match_reference_semantics(cuda):
    """Calling the returned closure step by step (``t = i*dt``) equals one run."""
    st = make_stage("real", a=10, static="1/2", dynamic="t/4")
    init = plane_wave(st)
    st.psi = torch.from_numpy(init).cuda()
    for i in range(st.steps):
        out = st.propagator(st, i * st.dt)
        assert out is st.psi
    a = st.psi.cpu().numpy()
    st.psi = torch.from_numpy(init).cuda()
    st.propagator.run(st, st.steps, 0)
    np.testing.assert_allclose(a, st.psi.cpu().numpy(), rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("kind,dynamic", [("imaginary", False), ("real", False), ("real", True)])
def test_spatial_expressions_at_each_grid_point(cuda, kind, dynamic):
    from gpe_simulator_b200.make_propagator import make_imag_spatial_kernel, make_real_spatial_kernel
    st = make_stage(kind, n=7, static="x/2 + y**2/10 + abs(z)/5",
                    dynamic="sin(t)*x + cos(pi)*z" if dynamic else None)
    st.psi.fill_(0.2 + 0.1j)
    x = st.x_array.cpu().numpy()
    X, Y, Z = x[:, None, None], x[None, :, None], x[None, None, :]
    pot = X / 2 + Y ** 2 / 10 + np.abs(Z) / 5
    t = 0.37
    if dynamic:
        pot = pot + np.sin(t) * X - Z
    kern = make_imag_spatial_kernel(st) if kind == "imaginary" else make_real_spatial_kernel(st)
    kern(st.psi, t)
    expo = -pot * st.dt / 2 * (1 if kind == "imaginary" else 1j)
    np.testing.assert_allclose(st.psi.cpu().numpy(), (0.2 + 0.1j) * np.exp(expo), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("static", [False, True])
def test_imaginary_decay_and_normalisation(cuda, static):
    from gpe_simulator_b200.launch import launch_stage
    st = make_stage("imaginary", static="1/2" if static else None)
    low, high = plane_wave(st, 1), plane_wave(st, 2)
    st.psi = torch.from_numpy(low + high).cuda()
    T = st.steps * st.dt
    want = low * np.exp(-T) + high * np.exp(-4 * T)
    dx = float(st.x_array[1] - st.x_array[0])
    want /= np.sqrt(np.sum(np.abs(want) ** 2) * dx ** 3)
    np.testing.assert_allclose(launch_stage(st).cpu().numpy(), want, rtol=1e-11, atol=1e-12)


def test_absorber_keeps_analytic_norm_loss(cuda):
    from gpe_simulator_b200.helper import get_N
    from gpe_simulator_b200.launch import launch_stage
    st = make_stage("real")
    init = plane_wave(st)
    st.psi = torch.from_numpy(init).cuda()
    gamma = 0.4
    st.staticV.fill_(-1j * gamma)
    T = st.steps * st.dt
    res = launch_stage(st)
    np.testing.assert_allclose(res.cpu().numpy(), init * np.exp((-gamma - 1j) * T), rtol=1e-11, atol=1e-12)
    assert abs(get_N(res, st.x_array) - np.exp(-2 * gamma * T)) < 1e-11


def test_cutoff_removes_high_mode_without_renormalising(cuda):
    from gpe_simulator_b200.helper import get_N
    from gpe_simulator_b200.launch import launch_stage
    st = make_stage("real", k_cut=1.5)
    low, high = plane_wave(st, 1), plane_wave(st, 2)
    st.psi = torch.from_numpy((low + high) / np.sqrt(2)).cuda()
    res = launch_stage(st)
    want = low * np.exp(-1j * st.steps * st.dt) / np.sqrt(2)
    np.testing.assert_allclose(res.cpu().numpy(), want, rtol=1e-11, atol=1e-12)
    assert abs(get_N(res, st.x_array) - 0.5) < 1e-11


def test_input_validation_is_assertion_error(cuda):
    st = make_stage("real")
    st.psi = st.psi.to(torch.complex128)[:, :, :4]
    with pytest.raises(AssertionError):
        st.propagator(st)
    st2 = make_stage("imaginary")
    st2.staticV = st2.staticV.to(torch.complex128)
    with pytest.raises(AssertionError):
        st2.propagator(st2)


def test_scalar_plane_wave_diagnostics(cuda):
    """``tests/test_diagnostics.py:31-39``: N = 1 and E_kin = 14."""
    from gpe_simulator_b200 import helper
    n, L = 16, 2 * np.pi
    x, k = helper.get_grids(n, L)
    xs = x.cpu().numpy()
    ph = 2 * xs[:, None, None] - 3 * xs[None, :, None] + xs[None, None, :]
    psi = torch.from_numpy(np.exp(1j * ph) / L ** 1.5).cuda()
    assert helper.get_N(psi, x) == pytest.approx(1, abs=1e-12)
    assert helper.get_E(helper.fftn(psi, x), x, k) == pytest.approx(14, abs=1e-11)


def test_zero_mode_spectrum(cuda):
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.nk_extraction import nk_extraction
    x, k = helper.get_grids(8, 2 * np.pi)
    psi = torch.ones((8, 8, 8), dtype=torch.complex128, device="cuda") / (2 * np.pi) ** 1.5
    spec = nk_extraction(helper.fftn(psi, x), x, k)
    assert spec["Nk"][0] == pytest.approx(1)
    np.testing.assert_allclose(spec["Nk"][1:], 0, atol=1e-25)
    assert int(spec["counts"][0]) == 1


class DLArray:
    """A CUDA array that only exports DLPack, as the reference's CuPy arrays do."""

    def __init__(self, t):
        self.t = t

    def __dlpack__(self, *args, **kwargs):
        return self.t.__dlpack__(*args, **kwargs)

    def __dlpack_device__(self):
        return self.t.__dlpack_device__()


@pytest.mark.parametrize("kind", ["real", "imaginary"])
def test_closure_takes_dlpack_arrays_in_place(cuda, kind):
    """A stage holding foreign (DLPack) arrays is advanced in place, zero-copy,
    and the closure returns the caller's own psi object."""
    a = make_stage(kind, n=16, L=8.0, a=50.0, static="x**2+y**2+z**2",
                   dynamic="0.5*sin(t)*x" if kind == "real" else None)
    b = make_stage(kind, n=16, L=8.0, a=50.0, static="x**2+y**2+z**2",
                   dynamic="0.5*sin(t)*x" if kind == "real" else None)
    raw = b.psi.clone()
    b.psi, b.staticV = DLArray(raw), DLArray(b.staticV.clone())
    b.x_array, b.k_array = DLArray(b.x_array.clone()), DLArray(b.k_array.clone())
    for i in range(3):
        args = (i * a.dt,) if getattr(a.propagator, "dynamic", False) else ()
        a.psi = a.propagator(a, *args)
        out = b.propagator(b, *args)
        assert out is b.psi
    torch.cuda.synchronize()
    assert torch.equal(a.psi, raw)


@pytest.mark.parametrize("kind", ["imaginary", "real"])
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 2e-5)])
def test_exact_local_mode_matches_oracle(cuda, kind, dtype, tol):
    """The opt-in exact local sub-flows (imaginary time; real time with an
    absorber) against the oracle's restatement; the default stays the reference's."""
    from gpe_simulator_b200 import Plan
    from oracle import ssf
    from tests.golden import cases
    c = cases.LOSSY16
    n, L, expr = 16, 8.0, "0.5*x**2+0.5*y**2+z**2/4"
    x, k = ssf.get_grids(n, L)
    static_v = cases.lossy_potential(x, c) if kind == "real" else None
    kw = dict(dtype=dtype, kind=kind, beta=300.0, dt=2e-3, static_expr=expr)
    exact, plain = Plan(n, x, k, exact_local=True, **kw), Plan(n, x, k, **kw)
    if static_v is not None:
        for p in (exact, plain):
            p.set_static_potential(torch.from_numpy(static_v).cuda())
    psi0 = ssf.noisy_gaussian(x, seed=2)
    a = torch.from_numpy(psi0).to(dtype).cuda()
    b = a.clone()
    exact.step(a, 20, 0)
    plain.step(b, 20, 0)
    m = ssf.Model(n=n, simulation_range=L, kind=kind, beta=300.0, dt=2e-3, static_expr=expr,
                  static_v=static_v, exact_local=True)
    want = ssf.run(psi0, m, 20)
    assert ssf.rel_l2(a.cpu().numpy().astype(np.complex128), want) < tol
    # the default is the reference's frozen-density step (the two differ at second
    # order in beta |psi|^2 dt/2, so only a little at this step size)
    assert not torch.equal(a, b)
