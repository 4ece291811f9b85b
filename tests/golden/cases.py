"""Parameters of the golden cases (shared by the generator and the tests).

Every case is in reference units: kinetic factor ``exp(-i k^2 dt)``, local
factor ``exp(-i (V + beta |psi|^2) dt/2)``.  The oscillator-unit workloads map
onto them exactly with ``V_ref = 2 V``, ``beta = 2 g``, ``dt_ref = dt / 2``,
``t_ref = t / 2``.
"""

import numpy as np

TRAP = "x**2+1.44*y**2+2.25*z**2"   # 2 * (x^2 + 1.44 y^2 + 2.25 z^2)/2

GROUND64 = dict(n=64, L=16.0, beta=1000.0, dt=5e-4, static_expr=TRAP, seed=0,
                checkpoints=(100, 1000, 2000), sub=4)

STIR32 = dict(n=32, L=24.0, beta=2000.0, dt=2.5e-4, static_expr=TRAP, seed=1,
              imag_steps=200, checkpoints=(100, 400), sub=2,
              # beam in oscillator units: A=10, w=0.5, R=2, Omega 0 -> 0.5 over 200 steps
              amp=10.0, width=0.5, radius=2.0, omega=0.5, ramp_steps=200)

LOSSY16 = dict(n=16, L=8.0, beta=300.0, dt=2e-3, static_expr="0.5*x**2+0.5*y**2+z**2/4",
               dynamic_expr="0.3*sin(5*t)*x", k_cut=4.0, seed=2, steps=60,
               gamma=2.0, reach=1.0, wall=0.7, depth=5.0)

BOX24 = dict(n=24, L=12.0, beta=150.0, dt=1e-3, static_expr="0.2*(x*x+y*y)", seed=3,
             steps=100, R=3.0, length=8.0, wall=0.5, depth=10.0)

DIAG_SIZES = ((2, 2 * np.pi), (7, 2 * np.pi), (8, 2 * np.pi), (18, 2 * np.pi), (32, 10.0))
PROJ_SIZES = ((16, 8.0), (15, 6.0))


def stir_beam():
    """The STIR32 beam in reference units (amp x2, rates x2, ramp time /2)."""
    from oracle.ssf import Beam
    c = STIR32
    return Beam(amp=2 * c["amp"], width=c["width"], radius=c["radius"],
                omega=2 * c["omega"], t_ramp=c["ramp_steps"] * c["dt"])


def projections(psi, count=4, seed=1234):
    """Inner products of psi with fixed seeded real fields (touches every point)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        r = rng.standard_normal(psi.shape)
        out.append(np.sum(np.asarray(psi, np.complex128) * r))
    return np.array(out)


def lossy_potential(x, c):
    """Complex ``U - i Gamma``: a Gaussian wall in x plus an absorber ramp."""
    X, Y, Z = x[:, None, None], x[None, :, None], x[None, None, :]
    half = x[-1] - x[0]
    edge = np.maximum(c["reach"] - (half / 2 + 0.5 * (x[1] - x[0]) - np.abs(X)), 0) + 0 * Y + 0 * Z
    wall = c["depth"] * np.exp(-(np.abs(Y) - 2.5) ** 2 / (2 * c["wall"] ** 2)) + 0 * X + 0 * Z
    return np.ascontiguousarray(wall - 1j * c["gamma"] * edge, dtype=np.complex128)


def box_potential(x, c):
    """Real float64 array: cylinder walls plus end caps (``gpe/potentials.py:3-11`` form)."""
    X, Y, Z = x[:, None, None], x[None, :, None], x[None, None, :]
    tube = np.exp(-(np.sqrt(X ** 2 + Y ** 2) - c["R"]) ** 2 / (2 * c["wall"] ** 2))
    sheet = np.exp(-(np.abs(Z) - c["length"] / 2) ** 2 / (2 * c["wall"] ** 2))
    return np.ascontiguousarray(c["depth"] * np.maximum(tube, sheet), dtype=np.float64)


def diag_state(n, seed=42):
    """Seeded complex normal state (``tests/test_diagnostics.py:24-28`` form)."""
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, n, n)) + 1j * rng.normal(size=(n, n, n))
