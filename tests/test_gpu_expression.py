"""Time-dependent potentials written in the reference's expression grammar.

In the reference a stirring beam is a user expression in ``x, y, z, t``
spliced into the half-step kernel and evaluated at ``t_mid`` in both halves
(``gpe/make_kernel.py:14-45``, ``gpe/make_propagator.py:86-103``).  Here an
expression none of whose additive terms depends on z runs on the
register-resident sweeps: the host folds its time-dependent subexpressions into
per-launch slot values and the z sweeps evaluate the rest once per z-line.
These tests check that such an expression (the rotating beam with a linear
ramp of its rate, written with ``abs`` as the reference grammar allows) takes
that path, agrees with the built-in beam and with the generic sweeps, and that
an expression with a z-dependent time term still runs (on the generic sweeps)
and matches the oracle.
"""

import numpy as np
import pytest
import torch

from oracle import ssf

pytestmark = pytest.mark.gpu

TRAP = "x**2+1.44*y**2+2.25*z**2"


def beam_ref(dt):
    """The bench beam (A = 10, w = 0.5, R = 2, rate 0 -> 0.5 over 200 steps of dt) in
    reference units, as ``oracle.ssf.Beam`` (which renders the grammar form)."""
    return ssf.Beam(amp=20.0, width=0.5, radius=2.0, omega=1.0, t_ramp=200 * dt / 2)


def plans(n, L, dtype, dt, **kw):
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, L)
    return Plan(n, x, k, dtype=dtype, kind="real", beta=4000.0, dt=dt / 2, static_expr=TRAP, **kw), x


def start_state(n, L, dtype, seed=3):
    from gpe_simulator_b200 import Plan
    x, k = ssf.get_grids(n, L)
    relax = Plan(n, x, k, dtype=torch.complex128, kind="imaginary", beta=4000.0, dt=2.5e-4, static_expr=TRAP)
    psi = torch.from_numpy(ssf.noisy_gaussian(x, seed=seed)).cuda()
    relax.step(psi, 100)
    relax.close()
    return psi.to(dtype).contiguous()


def rel(a, b):
    d = a.to(torch.complex128) - b.to(torch.complex128)
    return float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b.to(torch.complex128)))


# complex64: the two forms round the beam differently in the last bit of the
# per-line potential, which the state's complex64 rounding noise then carries
# (5e-6 after 300 steps, like complex64 against complex128)
@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_grammar_beam_runs_on_register_resident_sweeps_like_builtin(cuda, dtype, tol):
    from gpe_simulator_b200 import Beam
    from gpe_simulator_b200.plan import launch_count
    n, L, dt = 128, 24.0, 2.5e-4
    b = beam_ref(dt)
    expr_plan, _ = plans(n, L, dtype, dt, dynamic_expr=b.expression())
    builtin, _ = plans(n, L, dtype, dt, beam=Beam(b.amp, b.width, b.radius, b.omega, b.t_ramp))
    a = start_state(n, L, dtype)
    c = a.clone()
    before = launch_count(expr_plan)
    expr_plan.step(a, 300, 0)
    # register-resident real-time steps: a first z sweep, then 4 sweeps per step,
    # each z sweep preceded by the launch that tabulates the line terms
    assert launch_count(expr_plan) - before == 2 + 5 * 300
    builtin.step(c, 300, 0)
    assert rel(a, c) < tol
    # diagnostics on the same path (the potential energy takes the line terms)
    t = 300 * dt / 2
    da, dc = expr_plan.diagnostics(a, t=t), builtin.diagnostics(c, t=t)
    for key in ("N", "E_pot", "E"):
        assert abs(da[key] - dc[key]) <= 1e-5 * abs(dc[key]), (key, da[key], dc[key])


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_line_form_matches_generic_sweeps(cuda, dtype, tol):
    """A line-form expression with several time terms (rotating beam, a t-only
    offset, a modulated tilt in x) against the generic sweeps' per-point bytecode."""
    n, L, dt = 64, 16.0, 5e-4
    expr = beam_ref(dt).expression() + "+0.5*sin(3*t)+0.2*cos(t)*x-0.1*y*t"
    fast, _ = plans(n, L, dtype, dt, dynamic_expr=expr)
    generic, _ = plans(n, L, dtype, dt, dynamic_expr=expr, generic_only=True)
    a = start_state(n, L, dtype, seed=5)
    c = a.clone()
    fast.step(a, 200, 0)
    generic.step(c, 200, 0)
    assert rel(a, c) < tol
    for s in range(3):                    # per-step closure calls at arbitrary times
        fast.step_at(a, 0.37 + s * 0.01)
        generic.step_at(c, 0.37 + s * 0.01)
    assert rel(a, c) < tol


def test_z_dependent_time_term_falls_back_and_matches_oracle(cuda):
    from gpe_simulator_b200.plan import launch_count
    n, L, dt = 32, 12.0, 1e-3
    expr = "0.5*sin(4*t)*z**2+0.3*x*z*cos(t)"
    plan, x = plans(n, L, torch.complex128, dt, dynamic_expr=expr)
    psi0 = ssf.noisy_gaussian(x, seed=9)
    psi = torch.from_numpy(psi0.copy()).cuda()
    before = launch_count(plan)
    plan.step(psi, 20, 0)
    assert launch_count(plan) - before == 5 * 20     # generic: 5 sweeps per step
    m = ssf.Model(n=n, simulation_range=L, kind="real", beta=4000.0, dt=dt / 2, static_expr=TRAP,
                  dynamic_expr=expr)
    want = ssf.run(psi0, m, 20)
    assert ssf.rel_l2(psi.cpu().numpy(), want) < 1e-12
