"""The CPU oracle pinned against the reference: its analytic checks and the
fixtures generated by running the reference's own code (``tests/golden``)."""

import math
from pathlib import Path

import numpy as np
import pytest

from oracle import expr, ssf
from tests.golden import cases

GOLD = Path(__file__).resolve().parent / "golden"


def plane(x, mode=1):
    n = len(x)
    return np.broadcast_to(np.exp(1j * mode * x)[:, None, None], (n,) * 3).copy() / (2 * np.pi) ** 1.5


@pytest.mark.parametrize("static", [False, True])
@pytest.mark.parametrize("dynamic", [False, True])
@pytest.mark.parametrize("cutoff", [False, True])
def test_real_phase_kat(static, dynamic, cutoff):
    """``tests/test_propagators.py:61-84`` of the reference."""
    beta = ssf.get_beta(150000, 10)
    m = ssf.Model(n=8, simulation_range=2 * np.pi, kind="real", beta=beta, dt=0.01,
                  static_expr="1/2" if static else "0", dynamic_expr="t/4" if dynamic else "0",
                  k_cut=1.5 if cutoff else None)
    init = plane(m.x)
    out = ssf.run(init, m, 3)
    T = 0.03
    phase = (1 + beta / (2 * np.pi) ** 3) * T + (0.5 * T if static else 0) + (T ** 2 / 8 if dynamic else 0)
    np.testing.assert_allclose(out, init * np.exp(-1j * phase), rtol=1e-11, atol=1e-12)
    assert ssf.get_N(out, m.x) == pytest.approx(1, abs=1e-11)


def test_imaginary_two_mode_decay():
    m = ssf.Model(n=8, simulation_range=2 * np.pi, kind="imaginary", beta=0.0, dt=0.01, static_expr="1/2")
    low, high = plane(m.x, 1), plane(m.x, 2)
    out = ssf.run(low + high, m, 3)
    want = low * np.exp(-0.03) + high * np.exp(-0.12)
    want /= np.sqrt(np.sum(np.abs(want) ** 2) * m.dx ** 3)
    np.testing.assert_allclose(out, want, rtol=1e-11, atol=1e-12)


def test_absorber_and_cutoff():
    m = ssf.Model(n=8, simulation_range=2 * np.pi, kind="real", beta=0.0, dt=0.01,
                  static_v=np.full((8, 8, 8), -0.4j))
    init = plane(m.x)
    np.testing.assert_allclose(ssf.run(init, m, 3), init * np.exp((-0.4 - 1j) * 0.03), rtol=1e-11, atol=1e-12)
    m = ssf.Model(n=8, simulation_range=2 * np.pi, kind="real", beta=0.0, dt=0.01, k_cut=1.5)
    low, high = plane(m.x, 1), plane(m.x, 2)
    out = ssf.run((low + high) / np.sqrt(2), m, 3)
    np.testing.assert_allclose(out, low * np.exp(-0.03j) / np.sqrt(2), rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_spatial_expression_halfstep(kind):
    m = ssf.Model(n=7, simulation_range=2 * np.pi, kind=kind, beta=0.0, dt=0.01,
                  static_expr="x/2 + y**2/10 + abs(z)/5",
                  dynamic_expr="sin(t)*x + cos(pi)*z" if kind == "real" else "0")
    psi = np.full((7, 7, 7), 0.2 + 0.1j)
    X, Y, Z = m.axes()
    pot = X / 2 + Y ** 2 / 10 + np.abs(Z) / 5
    if kind == "real":
        pot = pot + np.sin(0.37) * X - Z
    ssf.halfstep(psi, m, 0.37)
    expo = -pot * 0.005 * (1 if kind == "imaginary" else 1j)
    np.testing.assert_allclose(psi, (0.2 + 0.1j) * np.exp(expo), rtol=1e-12, atol=1e-12)


def test_plane_wave_energy_kat():
    """``tests/test_diagnostics.py:31-39``: N = 1, E_kin = 14."""
    x, k = ssf.get_grids(16, 2 * np.pi)
    ph = 2 * x[:, None, None] - 3 * x[None, :, None] + x[None, None, :]
    psi = np.exp(1j * ph) / (2 * np.pi) ** 1.5
    assert ssf.get_N(psi, x) == pytest.approx(1, abs=1e-12)
    assert ssf.get_E(np.fft.fftn(psi), x, k) == pytest.approx(14, abs=1e-11)


@pytest.mark.parametrize("n,L", cases.DIAG_SIZES)
def test_diagnostics_against_reference_fixtures(n, L):
    g = np.load(GOLD / f"diag_n{n}.npz")
    x, k = ssf.get_grids(n, L)
    psi = cases.diag_state(n)
    F = np.fft.fftn(psi)
    assert ssf.get_N(psi, x) == pytest.approx(float(g["N"]), rel=1e-13)
    assert ssf.get_E(F, x, k) == pytest.approx(float(g["E_kin"]), rel=1e-13)
    spec = ssf.nk_extraction(F, x, k)
    for key in ("k", "counts", "edges", "complete_shells"):
        np.testing.assert_array_equal(spec[key], g[f"nk_{key}"])
    np.testing.assert_allclose(spec["Nk"], g["nk_Nk"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(spec["nk"], g["nk_nk"], rtol=1e-12, atol=1e-14)
    # Parseval (``tests/test_diagnostics.py:52-72``)
    assert spec["Nk"].sum() == pytest.approx(ssf.get_N(psi, x), rel=1e-12)
    assert spec["counts"].sum() == n ** 3
    # angular momentum (reference get_L, slab size 3 in the fixture; the sum is slab-independent)
    assert ssf.get_L(psi, x, k, slab_size=5) == pytest.approx(float(g["L"]), rel=1e-11, abs=1e-11)


@pytest.mark.parametrize("charge", [-1, 1])
def test_vortex_angular_momentum(charge):
    """``tests/test_diagnostics.py:40-48``: a charge-q vortex carries Lz = q N."""
    x, k = ssf.get_grids(48, 16.0)
    X, Y, Z = x[:, None, None], x[None, :, None], x[None, None, :]
    psi = (X + charge * 1j * Y) * np.exp(-(X * X + Y * Y + Z * Z) / 2)
    N = ssf.get_N(psi, x)
    assert ssf.get_L(psi, x, k, slab_size=7) == pytest.approx(charge * N, rel=1e-9, abs=1e-10)


def test_ground_state_fixture_first_checkpoint():
    c = cases.GROUND64
    g = np.load(GOLD / "ground64.npz")
    m = ssf.Model(n=c["n"], simulation_range=c["L"], kind="imaginary", beta=c["beta"], dt=c["dt"],
                  static_expr=c["static_expr"])
    psi = ssf.run(ssf.noisy_gaussian(m.x, seed=c["seed"]), m, 100)
    assert ssf.rel_l2(psi[::4, ::4, ::4], g["psi_sub_100"]) < 1e-13
    assert ssf.get_N(psi, m.x) == pytest.approx(float(g["N_100"]), rel=1e-14)
    assert ssf.get_E(np.fft.fftn(psi), m.x, m.k) == pytest.approx(float(g["E_kin_100"]), rel=1e-12)


def test_stirring_fixture_expression_and_builtin_beam():
    """The oracle's built-in beam and the beam as a reference expression agree with
    the reference run (first checkpoint)."""
    c = cases.STIR32
    g = np.load(GOLD / "stir32.npz")
    imag = ssf.Model(n=c["n"], simulation_range=c["L"], kind="imaginary", beta=c["beta"], dt=c["dt"],
                     static_expr=c["static_expr"])
    psi0 = ssf.run(ssf.noisy_gaussian(imag.x, seed=c["seed"]), imag, c["imag_steps"])
    assert ssf.rel_l2(psi0[::2, ::2, ::2], g["psi_start"]) < 1e-13
    mark = c["checkpoints"][0]
    b = cases.stir_beam()
    builtin = ssf.Model(n=c["n"], simulation_range=c["L"], kind="real", beta=c["beta"], dt=c["dt"],
                        static_expr=c["static_expr"], beam=b)
    text = ssf.Model(n=c["n"], simulation_range=c["L"], kind="real", beta=c["beta"], dt=c["dt"],
                     static_expr=c["static_expr"], dynamic_expr=b.expression())
    for model in (builtin, text):
        out = ssf.run(psi0, model, mark)
        assert ssf.rel_l2(out[::2, ::2, ::2], g[f"psi_sub_{mark}"]) < 1e-12


def test_lossy_and_box_fixtures():
    c = cases.LOSSY16
    x, _ = ssf.get_grids(c["n"], c["L"])
    m = ssf.Model(n=c["n"], simulation_range=c["L"], kind="real", beta=c["beta"], dt=c["dt"],
                  static_expr=c["static_expr"], dynamic_expr=c["dynamic_expr"], k_cut=c["k_cut"],
                  static_v=cases.lossy_potential(x, c))
    out = ssf.run(ssf.noisy_gaussian(x, sigma=1.5, seed=c["seed"]), m, c["steps"])
    assert ssf.rel_l2(out, np.load(GOLD / "lossy16.npz")["psi"]) < 1e-13
    c = cases.BOX24
    x, _ = ssf.get_grids(c["n"], c["L"])
    m = ssf.Model(n=c["n"], simulation_range=c["L"], kind="imaginary", beta=c["beta"], dt=c["dt"],
                  static_expr=c["static_expr"], static_v=cases.box_potential(x, c))
    out = ssf.run(ssf.noisy_gaussian(x, sigma=2.0, seed=c["seed"]), m, c["steps"])
    assert ssf.rel_l2(out, np.load(GOLD / "box24.npz")["psi"]) < 1e-13


def test_oscillator_units_map_exactly_onto_reference_units():
    """c_kin = 1/2 with (V, g, dt) equals the reference convention with (2V, 2g, dt/2)."""
    n, L = 16, 8.0
    osc = ssf.Model(n=n, simulation_range=L, kind="real", beta=300.0, dt=2e-3, ckin=0.5,
                    static_expr="0.5*(x**2+1.44*y**2+2.25*z**2)")
    ref = ssf.Model(n=n, simulation_range=L, kind="real", beta=600.0, dt=1e-3, ckin=1.0,
                    static_expr="x**2+1.44*y**2+2.25*z**2")
    psi = ssf.noisy_gaussian(osc.x, seed=3)
    assert ssf.rel_l2(ssf.run(psi, osc, 20), ssf.run(psi, ref, 20)) < 1e-13


def test_energies_consistent_with_reference_kinetic_energy():
    m = ssf.Model(n=16, simulation_range=8.0, kind="imaginary", beta=100.0, dt=1e-3,
                  static_expr="x**2+y**2+z**2")
    psi = ssf.noisy_gaussian(m.x, seed=4)
    e = ssf.energies(psi, m)
    assert e["E_kin"] == pytest.approx(ssf.get_E(np.fft.fftn(psi), m.x, m.k), rel=1e-14)
    assert e["E"] == pytest.approx(e["E_kin"] + e["E_pot"] + e["E_int"])
    assert e["mu"] == pytest.approx((e["E_kin"] + e["E_pot"] + 2 * e["E_int"]) / e["N"])


def test_expression_evaluator_grammar():
    X = np.array([0.5])
    assert expr.evaluate("x**2 + abs(-y) + pi", X, 2.0, 0.0)[0] == pytest.approx(0.25 + 2 + math.pi)
    assert expr.evaluate("sin(t)*x", X, 0, 0, t=1.0, time_dependent=True)[0] == pytest.approx(0.5 * math.sin(1))
    for bad in ("t*y", "x; 0", "foo(x)", "x^2"):
        with pytest.raises((ValueError, SyntaxError)):
            expr.evaluate(bad, X, 0, 0)


@pytest.mark.parametrize("n,L", cases.PROJ_SIZES)
def test_projections_against_reference_save_outputs(n, L):
    """TOF and density images as the reference's save_outputs writes them."""
    g = np.load(GOLD / f"proj_n{n}.npz")
    x, k = ssf.get_grids(n, L)
    out = ssf.projections(cases.diag_state(n, seed=7), x, k)
    for key in ssf.PROJECTIONS:
        np.testing.assert_array_equal(np.isnan(out[key]), np.isnan(g[key]))
        np.testing.assert_allclose(np.nan_to_num(out[key]), np.nan_to_num(g[key]), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("kind", ["imaginary", "real"])
def test_exact_local_flow_is_the_limit_of_frozen_density_substeps(kind):
    """The exact local sub-flow (an opt-in accuracy mode) equals the limit of
    many frozen-density micro-steps of the same local equation, with the trap
    and, in real time, an absorber U - i Gamma."""
    n, L = 8, 8.0
    x, _ = ssf.get_grids(n, L)
    X, Y, Z = x[:, None, None], x[None, :, None], x[None, None, :]
    static_v = None
    if kind == "real":
        static_v = (0.3 * X ** 2 - 1j * (0.8 + 0.5 * np.tanh(Y))).astype(np.complex128) * np.ones((n, n, n))
    kw = dict(n=n, simulation_range=L, kind=kind, beta=900.0, dt=0.02, static_expr="x**2+2*y**2+0.5*z**2",
              static_v=static_v)
    psi0 = ssf.noisy_gaussian(x, seed=2)
    exact = ssf.halfstep(psi0.copy(), ssf.Model(exact_local=True, **kw))
    micro = ssf.Model(**{**kw, "dt": kw["dt"] / 4000})
    fine = psi0.copy()
    for _ in range(4000):
        ssf.halfstep(fine, micro)
    assert ssf.rel_l2(exact, fine) < 2e-4          # first order in the micro step
    plain = ssf.halfstep(psi0.copy(), ssf.Model(**kw))
    assert ssf.rel_l2(exact, fine) < 0.05 * ssf.rel_l2(plain, fine)


def test_exact_local_closed_forms_for_uniform_states():
    n, L, beta, dt = 4, 4.0, 50.0, 0.1
    h = dt / 2
    c = 0.3 + 0.2j
    rho = abs(c) ** 2
    psi = np.full((n, n, n), c)
    m = ssf.Model(n=n, simulation_range=L, kind="imaginary", beta=beta, dt=dt, exact_local=True)
    np.testing.assert_allclose(ssf.halfstep(psi.copy(), m), c / np.sqrt(1 + 2 * beta * rho * h), rtol=1e-14)
    g = 0.7
    m = ssf.Model(n=n, simulation_range=L, kind="real", beta=beta, dt=dt, exact_local=True,
                  static_v=np.full((n, n, n), -1j * g))
    tau = -np.expm1(-2 * g * h) / (2 * g)
    np.testing.assert_allclose(ssf.halfstep(psi.copy(), m), c * np.exp(-g * h - 1j * beta * rho * tau), rtol=1e-14)
