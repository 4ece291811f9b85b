"""Batched solves: each instance's result is the same alone and in the batch."""

import numpy as np
import pytest
import torch

from oracle import ssf

pytestmark = pytest.mark.gpu


def small_batch():
    from gpe_simulator_b200.batch import Instance
    # mixed sizes: register-resident (48, 64, 96, 128) and generic (18)
    specs = [(48, 12.0, 300.0, "x**2+y**2+z**2"), (64, 12.0, 800.0, "x**2+1.44*y**2+2.25*z**2"),
             (18, 8.0, 50.0, "x**2+0.5*y**2+2*z**2"), (64, 16.0, 1200.0, "x**2+y**2+4*z**2"),
             (96, 14.0, 2000.0, "x**2+2*y**2+z**2"), (128, 16.0, 500.0, "x**2+y**2+z**2")]
    return [Instance(n=n, simulation_range=L, beta=b, dt=5e-4, static_expr=e) for n, L, b, e in specs]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_batch_equals_one_at_a_time_bitwise(cuda, dtype):
    from gpe_simulator_b200 import Plan
    from gpe_simulator_b200.batch import Batch, initial_states
    insts = small_batch()
    states = initial_states(insts, dtype)
    alone = []
    for inst, psi in zip(insts, states):
        p = Plan(inst.n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                 static_expr=inst.static_expr)
        a = psi.clone()
        p.step(a, 25)
        alone.append(a)
    b = Batch(insts, dtype)
    mixed = [s.clone() for s in states]
    b.bind(mixed)
    b.step(25)
    torch.cuda.synchronize()
    for a, m in zip(alone, mixed):
        assert torch.equal(a, m)
    # a subset (active mask) keeps the others untouched and still matches
    before = [m.clone() for m in mixed]
    b.bind(mixed, active=[1, 0, 1, 0, 1, 0])
    b.step(3)
    torch.cuda.synchronize()
    for i, (m, s) in enumerate(zip(mixed, before)):
        assert torch.equal(m, s) == (i % 2 == 1)


def test_batch_matches_oracle(cuda):
    from gpe_simulator_b200.batch import Batch, initial_states
    insts = small_batch()[:3]
    states = initial_states(insts, torch.complex128)
    b = Batch(insts, torch.complex128)
    work = [s.clone() for s in states]
    b.bind(work)
    b.step(30)
    for inst, s, w in zip(insts, states, work):
        m = ssf.Model(n=inst.n, simulation_range=inst.simulation_range, kind="imaginary", beta=inst.beta,
                      dt=inst.dt, static_expr=inst.static_expr)
        want = ssf.run(s.cpu().numpy(), m, 30)
        assert ssf.rel_l2(w.cpu().numpy(), want) < 1e-12
    diag = b.diagnostics()
    for inst, w, d in zip(insts, work, diag):
        m = ssf.Model(n=inst.n, simulation_range=inst.simulation_range, kind="imaginary", beta=inst.beta,
                      dt=inst.dt, static_expr=inst.static_expr)
        e = ssf.energies(w.cpu().numpy(), m)
        assert d[0] == pytest.approx(e["N"], rel=1e-12)
        assert d[4] == pytest.approx(e["E"], rel=1e-10)
        assert d[5] == pytest.approx(e["mu"], rel=1e-10)


def test_solve_converges_and_retires(cuda):
    from gpe_simulator_b200.batch import Batch, initial_states
    insts = small_batch()[:4]
    b = Batch(insts, torch.complex64)
    states = initial_states(insts, torch.complex64)
    steps, final = b.solve(states, tol=1e-6, max_steps=3000, check_every=20)
    assert (steps > 0).all() and (steps <= 3000).all()
    assert np.isfinite(final).all()
    np.testing.assert_allclose(final[:, 0], 1.0, atol=1e-5)


def _host_checked_solve(b, states, tol, max_steps, chunk):
    """The convergence loop on the host: step(chunk) + diagnostics per check,
    converged instances unbound at once (the rule gpe_batch_run applies on the device)."""
    count = len(states)
    b.bind(states, np.ones(count, np.int32))
    steps = np.zeros(count, np.int64)
    last = b.diagnostics()[:, 4]
    done = np.zeros(count, bool)
    final = np.full((count, 6), np.nan)
    while not done.all():
        b.step(chunk)
        steps[~done] += chunk
        diag = b.diagnostics()
        e = diag[:, 4]
        with np.errstate(invalid="ignore", divide="ignore"):
            rate = np.abs(e - last) / (chunk * np.abs(e))
        newly = (~done) & ((rate < tol) | (steps >= max_steps))
        final[newly] = diag[newly]
        last = np.where(done, last, e)
        done |= newly
        if newly.any() and not done.all():
            b.bind(states, (~done).astype(np.int32))
    return steps, final


@pytest.mark.parametrize("checks_per_call", [1, 3, 8])
def test_device_convergence_equals_host_checks_bitwise(cuda, checks_per_call):
    """Batch.solve with the energy checks on the device (gpe_batch_run, several
    checks per synchronisation, converged instances frozen in place) stops every
    instance at the same step, with the same state and diagnostics bit for bit,
    as the host loop of step + diagnostics that unbinds each at its check."""
    from gpe_simulator_b200.batch import Batch, initial_states
    insts = small_batch()
    states = initial_states(insts, torch.complex64)
    # tolerance from a probe run: the median of the instances' rates at the last
    # check, so that some converge before the cap and some run to it
    probe = Batch(insts, torch.complex64)
    c = [s.clone() for s in states]
    probe.bind(c)
    last = probe.diagnostics()[:, 4]
    for _ in range(20):
        probe.step(20)
        e = probe.diagnostics()[:, 4]
        rate, last = np.abs(e - last) / (20 * np.abs(e)), e
    probe.close()
    tol = float(np.median(rate))
    a = [s.clone() for s in states]
    b = [s.clone() for s in states]
    ba = Batch(insts, torch.complex64)
    steps_a, final_a = ba.solve(a, tol=tol, max_steps=400, check_every=20, checks_per_call=checks_per_call)
    bb = Batch(insts, torch.complex64)
    steps_b, final_b = _host_checked_solve(bb, b, tol=tol, max_steps=400, chunk=20)
    torch.cuda.synchronize()
    assert np.array_equal(steps_a, steps_b)
    assert (steps_a < 400).any() and (steps_a == 400).any()    # some stop early, some at the cap
    assert np.array_equal(final_a, final_b)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    ba.close()
    bb.close()


def test_batch_run_state_in_and_out(cuda):
    """gpe_batch_run's per-slot state: a frozen slot stays as it is, a live one
    advances by chunk per check, a NaN last energy blocks the first check, and the
    step cap freezes; gpe_batch_step afterwards still advances every bound instance."""
    from gpe_simulator_b200.batch import Batch, initial_states
    insts = small_batch()[:3]
    states = initial_states(insts, torch.complex64)
    b = Batch(insts, torch.complex64)
    b.bind(states)
    frozen = states[1].clone()
    live = np.array([1, 0, 1], np.int32)
    steps = np.array([0, 7, 40], np.int64)
    e_last = np.array([np.nan, 1.0, np.nan])
    diag = b.run(20, 3, 1e-30, 80, live, steps, e_last)
    torch.cuda.synchronize()
    assert steps.tolist() == [60, 7, 80] and live.tolist() == [1, 0, 0]
    assert e_last[1] == 1.0 and np.isfinite(e_last[[0, 2]]).all()
    assert torch.equal(states[1], frozen)
    assert np.isfinite(diag[[0, 2]]).all()
    before = states[1].clone()
    b.step(2)
    torch.cuda.synchronize()
    assert not torch.equal(states[1], before)
    with pytest.raises(ValueError, match="chunk"):
        b.run(0, 1, 1e-9, 20, live, steps, e_last)
    b.close()


def test_add_remove_keeps_results_identical(cuda):
    """Continuous batching: instances join and leave a running batch; every
    instance still matches its solo run bit for bit."""
    from gpe_simulator_b200 import Plan
    from gpe_simulator_b200.batch import Batch, Instance, initial_states
    insts = small_batch() + [Instance(n=32, simulation_range=8.0, beta=100.0, dt=5e-4,
                                      static_expr="x**2+y**2+z**2")]
    states = initial_states(insts, torch.complex64)
    plan_steps = {0: 40, 1: 20, 2: 60, 3: 20, 4: 40, 5: 20, 6: 20}
    alone = []
    for i, (inst, psi) in enumerate(zip(insts, states)):
        p = Plan(inst.n, inst.x, inst.k, dtype=torch.complex64, kind="imaginary", beta=inst.beta,
                 dt=inst.dt, static_expr=inst.static_expr)
        a = psi.clone()
        for _ in range(plan_steps[i] // 20):
            p.step(a, 20)
        alone.append(a)
    b = Batch([], torch.complex64)
    work = {}
    slots = {}
    schedule = [[0, 1, 2], [3, 4], [5, 6], [], [], []]   # joins per round
    done = {}
    for rnd, joins in enumerate(schedule):
        for i in joins:
            slots[i] = b.add(insts[i])
            work[i] = states[i].clone()
        psis = [None] * len(b.instances)
        for i, sl in slots.items():
            psis[sl] = work[i]
        b.bind(psis)
        b.step(20)
        b.diagnostics()
        for i in list(slots):
            done[i] = done.get(i, 0) + 20
            if done[i] >= plan_steps[i]:
                b.remove(slots.pop(i))
        if not slots and rnd >= 2:
            break
    torch.cuda.synchronize()
    for i in range(len(insts)):
        assert torch.equal(work[i], alone[i]), i


def test_serving_matches_one_at_a_time(cuda):
    """A short request stream: every imaginary-time result and every resident
    real-time state is identical whether served in the mix or alone."""
    from gpe_simulator_b200 import serve
    reqs = serve.workload(24, rate=400.0, seed=7)
    for r in reqs:
        if r.kind == "real":
            r.steps = min(r.steps, 300)
    s1 = serve.make_sessions(relax_steps=20)
    serve.Server(s1, chunk=20).run(reqs)
    reqs2 = serve.workload(24, rate=400.0, seed=7)
    for r in reqs2:
        if r.kind == "real":
            r.steps = min(r.steps, 300)
    s2 = serve.make_sessions(relax_steps=20)
    serve.run_plain(reqs2, s2, chunk=20)
    for a, b in zip(reqs, reqs2):
        assert a.taken == b.taken
        if a.kind == "imaginary":
            assert torch.equal(a.result["psi"], b.result["psi"])
            assert a.result["E"] == b.result["E"]
    for x, y in zip(s1, s2):
        assert x.step == y.step
        assert torch.equal(x.psi, y.psi)
    summary = serve.summarise(reqs)
    assert summary["requests"] == 24 and summary["p99_ms"] >= summary["p50_ms"] > 0


def test_serving_admits_by_free_device_memory(cuda):
    """Admission consults the device's free memory every round (a fake reading,
    injected on the host): with none free and nothing of its own running the
    server raises instead of waiting for ever; with room for one solve per round
    it defers the rest and still finishes every request."""
    from gpe_simulator_b200 import serve

    def solves():
        out = [r for r in serve.workload(12, rate=1000.0, seed=3) if r.kind == "imaginary"][:4]
        for r in out:
            r.arrival = 0.0          # all queued at once: one admission round sees them all
        return out

    total = 180 << 30
    with pytest.raises(MemoryError, match="free"):
        serve.Server([], mem_info=lambda: (0, total)).run(solves())
    one = serve.state_bytes(128, torch.complex64) + 1024
    srv = serve.Server([], mem_info=lambda: ((1 << 30) + one, total), reserve=1 << 30)
    reqs = solves()
    srv.run(reqs)
    assert srv.refused > 0
    assert all(r.done_at is not None and r.taken > 0 for r in reqs)


def test_real_time_stirring_sweep_batched_equals_alone_bitwise(cuda):
    """A stirring-rate sweep (rates 0.25/0.5/1 at two grid sizes and two g) batched
    with imaginary-time solves: every real-time state equals its own plan's
    one-step calls bit for bit, the clock carries the beam's time, and the
    diagnostics use the instance's current time."""
    from gpe_simulator_b200 import Plan
    from gpe_simulator_b200.batch import Batch, initial_states, stirring_instances, sweep_instances
    real = stirring_instances(rates=(0.25, 0.5, 1.0), gs=(500.0, 1000.0), grids=((32, 12.0), (64, 16.0)))
    imag = sweep_instances(3, seed=5)
    insts = real + imag
    states = initial_states(insts, torch.complex64, seed0=300)
    batch = Batch(insts, torch.complex64)
    work = [s.clone() for s in states]
    batch.bind(work)
    batch.set_step(1, 7)          # one instance starts further along its ramp
    batch.step(25)
    assert batch.get_step(1) == 32 and batch.get_step(0) == 25
    diag = batch.diagnostics()
    for i, inst in enumerate(insts):
        plan = Plan(inst.n, inst.x, inst.k, dtype=torch.complex64, kind=inst.kind, beta=inst.beta, dt=inst.dt,
                    static_expr=inst.static_expr, beam=inst.beam)
        alone = states[i].clone()
        s0 = 7 if i == 1 else 0
        if inst.kind == "real":
            for s in range(25):
                plan.step(alone, 1, s0 + s)      # one-step calls, as the batch runs them
        else:
            plan.step(alone, 25)
        assert torch.equal(alone, work[i]), (i, inst.kind, inst.n)
        d = plan.diagnostics(alone, t=(s0 + 25) * inst.dt if inst.kind == "real" else 0.0)
        assert np.allclose([d["N"], d["E"], d["mu"]], diag[i, [0, 4, 5]], rtol=1e-12, atol=0), i
        plan.close()
    batch.close()
