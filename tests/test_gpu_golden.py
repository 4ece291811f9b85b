"""CUDA path vs fixtures generated by running the reference itself.

The fixtures (``tests/golden/*.npz``, made by ``tests/golden/make_golden.py``)
hold the reference's own outputs (its propagator closures, kernel strings and
diagnostics, with numpy.fft in place of cuFFT).  complex128 must match to
1e-12 (psi relative L2); complex64 to 1e-5.
"""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import ssf
from tests.golden import cases

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLD / f"{name}.npz")


def rel(a, b):
    return ssf.rel_l2(a, b)


def plan_for(c, kind, dtype, **kw):
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(c["n"], c["L"])
    return Plan(c["n"], x, k, dtype=dtype, kind=kind, beta=c["beta"], dt=c["dt"],
                static_expr=c["static_expr"], **kw), x, k


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_ground_state_64(cuda, dtype, tol):
    c = cases.GROUND64
    g = load("ground64")
    plan, x, k = plan_for(c, "imaginary", dtype)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=c["seed"])).to(dtype).cuda()
    done = 0
    sub = c["sub"]
    for mark in c["checkpoints"]:
        plan.step(psi, mark - done, done)
        done = mark
        got = psi.cpu().numpy()
        err = rel(got[::sub, ::sub, ::sub], g[f"psi_sub_{mark}"])
        assert err < tol, (mark, err)
        # projections on seeded random fields touch every point (the subsample does not)
        proj = g[f"proj_{mark}"]
        perr = np.max(np.abs(cases.projections(got) - proj)) / np.max(np.abs(proj))
        assert perr < 10 * tol, (mark, perr)
        N = plan.norm(psi)
        assert abs(N - g[f"N_{mark}"]) < (1e-13 if dtype == torch.complex128 else 1e-6)


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 2e-5)])
def test_stirred_32(cuda, dtype, tol):
    from gpe_simulator_b200 import Plan
    c = cases.STIR32
    g = load("stir32")
    imag, x, k = plan_for(c, "imaginary", dtype)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=c["seed"])).to(dtype).cuda()
    imag.step(psi, c["imag_steps"])
    sub = c["sub"]
    assert rel(psi.cpu().numpy()[::sub, ::sub, ::sub], g["psi_start"]) < tol
    b = cases.stir_beam()
    from gpe_simulator_b200 import Beam
    real = Plan(c["n"], x, k, dtype=dtype, kind="real", beta=c["beta"], dt=c["dt"],
                static_expr=c["static_expr"],
                beam=Beam(b.amp, b.width, b.radius, b.omega, b.t_ramp))
    done = 0
    for mark in c["checkpoints"]:
        real.step(psi, mark - done, done)
        done = mark
        err = rel(psi.cpu().numpy()[::sub, ::sub, ::sub], g[f"psi_sub_{mark}"])
        assert err < tol, (mark, err)
        assert abs(real.norm(psi) - g[f"N_{mark}"]) < (1e-12 if dtype == torch.complex128 else 1e-6)


def test_stirred_32_expression_path(cuda):
    """The same beam written as a dynamic expression (device bytecode)."""
    from gpe_simulator_b200 import Plan
    c = cases.STIR32
    g = load("stir32")
    imag, x, k = plan_for(c, "imaginary", torch.complex128)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=c["seed"])).cuda()
    imag.step(psi, c["imag_steps"])
    real = Plan(c["n"], x, k, dtype=torch.complex128, kind="real", beta=c["beta"], dt=c["dt"],
                static_expr=c["static_expr"], dynamic_expr=cases.stir_beam().expression())
    real.step(psi, c["checkpoints"][0])
    err = rel(psi.cpu().numpy()[::2, ::2, ::2], g[f"psi_sub_{c['checkpoints'][0]}"])
    assert err < 1e-12, err


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_lossy_cutoff_16(cuda, dtype, tol):
    from gpe_simulator_b200 import Plan
    c = cases.LOSSY16
    g = load("lossy16")
    x, k = ssf.get_grids(c["n"], c["L"])
    plan = Plan(c["n"], x, k, dtype=dtype, kind="real", beta=c["beta"], dt=c["dt"],
                static_expr=c["static_expr"], dynamic_expr=c["dynamic_expr"], k_cut=c["k_cut"])
    plan.set_static_potential(torch.from_numpy(cases.lossy_potential(x, c)).cuda())
    psi = torch.from_numpy(ssf.noisy_gaussian(x, sigma=1.5, seed=c["seed"])).to(dtype).cuda()
    plan.step(psi, c["steps"])
    assert rel(psi.cpu().numpy(), g["psi"]) < tol
    assert abs(plan.norm(psi) - float(g["N"])) < 1e-6


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_box_potential_24(cuda, dtype, tol):
    from gpe_simulator_b200 import Plan
    c = cases.BOX24
    g = load("box24")
    x, k = ssf.get_grids(c["n"], c["L"])
    plan = Plan(c["n"], x, k, dtype=dtype, kind="imaginary", beta=c["beta"], dt=c["dt"],
                static_expr=c["static_expr"])
    plan.set_static_potential(torch.from_numpy(cases.box_potential(x, c)).cuda())
    psi = torch.from_numpy(ssf.noisy_gaussian(x, sigma=2.0, seed=c["seed"])).to(dtype).cuda()
    plan.step(psi, c["steps"])
    assert rel(psi.cpu().numpy(), g["psi"]) < tol


@pytest.mark.parametrize("n,L", cases.DIAG_SIZES)
def test_diagnostics_match_reference(cuda, n, L):
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.nk_extraction import nk_extraction
    g = load(f"diag_n{n}")
    x, k = helper.get_grids(n, L)
    psi = torch.from_numpy(cases.diag_state(n)).cuda()
    assert helper.get_N(psi, x) == pytest.approx(float(g["N"]), rel=1e-13)
    F = helper.fftn(psi, x)
    assert helper.get_E(F, x, k) == pytest.approx(float(g["E_kin"]), rel=1e-12)
    spec = nk_extraction(F, x, k)
    np.testing.assert_array_equal(spec["counts"], g["nk_counts"])
    np.testing.assert_allclose(spec["Nk"], g["nk_Nk"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(spec["nk"], g["nk_nk"], rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(spec["edges"], g["nk_edges"])
    np.testing.assert_array_equal(spec["k"], g["nk_k"])
    np.testing.assert_array_equal(spec["complete_shells"], g["nk_complete_shells"])
    # angular momentum: the reference's get_L on the same state
    assert helper.get_L(psi, x, k) == pytest.approx(float(g["L"]), rel=1e-10, abs=1e-10)


@pytest.mark.parametrize("charge", [-1, 1])
@pytest.mark.parametrize("dtype,rel", [(torch.complex128, 1e-9), (torch.complex64, 2e-5)])
def test_vortex_angular_momentum(cuda, charge, dtype, rel):
    """``tests/test_diagnostics.py:40-48``: a charge-q vortex carries Lz = q N."""
    from gpe_simulator_b200 import helper
    x, k = helper.get_grids(48, 16.0)
    xs = x.cpu().numpy()
    X, Y, Z = xs[:, None, None], xs[None, :, None], xs[None, None, :]
    psi = torch.from_numpy((X + charge * 1j * Y) * np.exp(-(X * X + Y * Y + Z * Z) / 2)).to(dtype).cuda()
    N = helper.get_N(psi, x)
    assert helper.get_L(psi, x, k, slab_size=7) == pytest.approx(charge * N, rel=rel, abs=1e-10)


@pytest.mark.parametrize("n,L", cases.PROJ_SIZES)
@pytest.mark.parametrize("dtype,rtol", [(torch.complex128, 1e-12), (torch.complex64, 2e-6)])
def test_projections_match_reference_save_outputs(cuda, n, L, dtype, rtol):
    """TOF columns and slices, column density, density slice and phase images as
    the reference's save_outputs writes them (even and odd n for fftshift)."""
    from gpe_simulator_b200 import Plan
    g = load(f"proj_n{n}")
    x, k = ssf.get_grids(n, L)
    plan = Plan(n, x, k, dtype=dtype, kind="imaginary", beta=0.0, dt=0.0)
    psi = torch.from_numpy(cases.diag_state(n, seed=7)).to(dtype).cuda()
    out = plan.projections(psi)
    assert list(out) == list(ssf.PROJECTIONS)
    for key in ssf.PROJECTIONS:
        want = g[key]
        np.testing.assert_array_equal(np.isnan(out[key]), np.isnan(want), err_msg=key)
        scale = np.nanmax(np.abs(want))
        np.testing.assert_allclose(np.nan_to_num(out[key]), np.nan_to_num(want), rtol=rtol,
                                   atol=(1e-12 if dtype == torch.complex128 else 2e-6) * scale, err_msg=key)
    sub = plan.projections(psi, ["phase_xy", "TOF_yz"])
    assert list(sub) == ["TOF_yz", "phase_xy"]
    assert np.array_equal(sub["TOF_yz"], out["TOF_yz"], equal_nan=True)


def test_stage_writes_reference_image_files(cuda, tmp_path):
    """launch_stage writes the reference's image files when their intervals are due."""
    from gpe_simulator_b200 import helper
    from gpe_simulator_b200.expressions import cuda_expression
    from gpe_simulator_b200.launch import launch_stage
    from gpe_simulator_b200.stage import stage
    n, L = 16, 8.0
    x, k = helper.get_grids(n, L)
    monitor = {key: 2 for key in ("show_TOF_image_interval", "show_verticle_TOF_interval",
                                  "show_TOF_slice_interval", "show_verticle_TOF_slice_interval",
                                  "show_magnifier_interval", "show_magnifier_slice_interval",
                                  "show_phase_interval")}
    st = stage(simulation_range=L, x_array=x, k_array=k, N_grids=n, type="imaginary", steps=4, dt=1e-3,
               initial_state=dict(type="gaussian", sigma=1.0), box_params=dict(activate=False),
               absorber_params=dict(activate=False), noise_params=dict(activate=False),
               cloud_params=dict(a=0.0, N_atom=1), monitor_params=monitor,
               save_params=dict(scalar_interval=0, nk_interval=0),
               potential_params=dict(static=dict(activate=True, expression=cuda_expression("x**2+y**2+z**2")),
                                     dynamic=dict(activate=False, expression="0")),
               k_cut_params=dict(activate=False, k_cut=0.0))
    st.prepare()
    st.monitor_dir = tmp_path
    psi = launch_stage(st)
    for name in ssf.PROJECTIONS:
        files = sorted(tmp_path.glob(f"{name}_*.npz"))
        assert [f.name for f in files] == [f"{name}_00000002.npz", f"{name}_00000004.npz"], name
    f = np.load(tmp_path / "TOF_xy_00000004.npz")
    want = ssf.projections(psi.cpu().numpy(), x.cpu().numpy(), k.cpu().numpy())["TOF_xy"]
    np.testing.assert_allclose(f["values"], want, rtol=1e-10, atol=1e-14)
    assert set(f.files) == {"step", "time", "values", "kx", "ky"}
