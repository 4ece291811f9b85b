"""Continuous-batching server for mixed imaginary-time and real-time requests.

Requests arrive over time (seeded Poisson process).  Each scheduling round the
server

1. admits the requests that have arrived, in arrival order, while the device
   memory a solve needs fits both the HBM budget and the memory the device
   reports free (queried every round) and, with a window (``max_active``), while
   fewer than that many requests run; a request that cannot start holds back
   the ones behind it, except a real-time segment whose session is still busy
   (its own earlier segments are ahead of it anyway);
2. advances all admitted work: the imaginary-time solves as one running
   :class:`Batch` (instances added on admission, removed on convergence) by
   ``checks_per_round`` chunks with the convergence test on the device (one
   synchronisation per round), and every real-time segment on its own CUDA
   stream, so the segments and the batch overlap on the device;
3. retires what finished (converged ground states, completed segments).

Real-time requests continue a device-resident state: the server keeps one
resident psi per session and each segment advances it in place by its number of
steps (segments of one session run in order).  Every request computes exactly
what it would compute alone (same kernels, same arithmetic), so results are
identical alone and in the mix.

``run_plain`` processes the same request stream one request at a time through
the single-plan path, for comparison.
"""

from dataclasses import dataclass, field
import math
import time

import numpy as np
import torch

from .batch import Batch, Instance, initial_states
from .plan import Beam, Plan, beam_in_reference_units

TRAP = "x**2+{ly}*y**2+{lz}*z**2"


@dataclass
class Request:
    rid: int
    arrival: float
    kind: str                  # "imaginary" | "real"
    inst: Instance = None      # imaginary: the solve
    tol: float = 1e-9
    max_steps: int = 5000
    session: int = -1          # real: resident state it continues
    steps: int = 0             # real: segment length
    done_at: float = None
    taken: int = 0
    result: dict = field(default_factory=dict)


@dataclass
class Session:
    """A device-resident real-time state and the plan that advances it."""
    n: int
    plan: Plan
    psi: torch.Tensor
    step: int = 0
    busy: bool = False


def workload(count=1000, rate=20.0, seed=2, imag_frac=0.7):
    """Seeded request stream: Poisson arrivals at ``rate`` per second; 70 % imaginary-time
    ground states (32^3-128^3, parameters drawn as in the batched sweep) and 30 %
    real-time stirring segments of 500-5000 steps continuing a resident state."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    imag_sizes = [(32, 5.0), (48, 6.0), (64, 8.0), (96, 10.0), (128, 12.0)]
    for rid in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.uniform() < imag_frac:
            n, L = imag_sizes[rng.integers(len(imag_sizes))]
            g = float(math.exp(rng.uniform(math.log(100.0), math.log(5000.0))))
            ly, lz = (float(v * v) for v in rng.uniform(0.5, 2.0, 2))
            inst = Instance(n=n, simulation_range=2 * L, beta=2 * g, dt=5e-4,
                            static_expr=TRAP.format(ly=repr(ly), lz=repr(lz)))
            out.append(Request(rid, t, "imaginary", inst=inst))
        else:
            out.append(Request(rid, t, "real", session=int(rng.integers(SESSIONS)),
                               steps=int(rng.integers(500, 5001))))
    return out


# resident real-time sessions: (grid side, box side) -- 64^3 to 256^3
SESSION_GRIDS = [(64, 16.0), (96, 18.0), (128, 20.0), (128, 24.0), (256, 24.0), (64, 12.0), (256, 24.0),
                 (128, 16.0)]
SESSIONS = len(SESSION_GRIDS)


def make_sessions(dtype=torch.complex64, relax_steps=200):
    """Resident states: each session's trap ground-state guess relaxed in imaginary time,
    then driven by the stirring beam (oscillator units A=10, w=0.5, R=2, Omega 0->0.5)."""
    out = []
    for s, (n, L) in enumerate(SESSION_GRIDS):
        inst = Instance(n=n, simulation_range=L, beta=2000.0, dt=5e-4, static_expr=TRAP.format(ly=1.44, lz=2.25))
        psi = initial_states([inst], dtype, seed0=500 + s)[0]
        prep = Plan(n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                    static_expr=inst.static_expr)
        prep.step(psi, relax_steps)
        prep.close()
        beam = beam_in_reference_units(10.0, 0.5, 2.0, 0.5, 200 * 2.5e-4)
        plan = Plan(n, inst.x, inst.k, dtype=dtype, kind="real", beta=inst.beta, dt=1.25e-4,
                    static_expr=inst.static_expr, beam=beam)
        out.append(Session(n=n, plan=plan, psi=psi))
    torch.cuda.synchronize()
    return out


def state_bytes(n, dtype):
    """Device memory a request holds: psi, the diagnostic work buffer, and tables."""
    esize = 8 if dtype == torch.complex64 else 16
    return 2 * n ** 3 * esize + 64 * n * 8 + (1 << 20)


class Server:
    """Continuous batching over a running imaginary-time :class:`Batch` and
    real-time segments on per-session streams (see the module docstring)."""

    def __init__(self, sessions, dtype=torch.complex64, budget=150e9, chunk=20, max_active=None,
                 mem_info=None, reserve=2 << 30, batch_priority=True, ordered=True, checks_per_round=16):
        self.sessions = sessions
        self.dtype = dtype
        self.budget = budget
        self.chunk = chunk
        # (free, total) bytes of the device; admission keeps `reserve` bytes free for
        # the allocator's own blocks and the plans' tables
        self.mem_info = mem_info or torch.cuda.mem_get_info
        self.reserve = reserve
        self.refused = 0       # admissions deferred because the device lacked free memory
        # at most this many requests run together (None: as many as the memory
        # budget admits); fewer finish sooner, more share each launch.  ordered:
        # the window counts imaginary-time solves and real-time segments alike and
        # admission keeps arrival order, so that under overload the device works
        # through the stream nearly first come, first served (a saturated device
        # then finishes the median request no later than one request at a time
        # would); otherwise the window counts solves only and segments start as
        # soon as their session is free.
        self.max_active = max_active
        self.ordered = ordered
        # energy checks (chunks) per scheduling round, run on the device: more keep
        # the device busy between host rounds, fewer admit arrivals sooner
        self.checks_per_round = checks_per_round
        # the imaginary-time batch advances in short chunks with a host check after
        # each, so it runs ahead of the long real-time segments: on the device's
        # highest stream priority (the batch's own streams follow it), segments at
        # the default priority
        self.streams = [torch.cuda.Stream() for _ in sessions]
        self.batch_stream = torch.cuda.Stream(priority=-100 if batch_priority else 0)

    def run(self, requests):
        """Serve ``requests`` against the wall clock (arrival times are offsets from the
        start); fills ``done_at`` (seconds since the start) and ``result``.  The
        imaginary-time requests share one tolerance and step cap (the batch's
        device-side check takes one of each)."""
        solves = [r for r in requests if r.kind == "imaginary"]
        if len({(r.tol, r.max_steps) for r in solves}) > 1:
            raise ValueError("imaginary-time requests of one run take one tol and max_steps")
        if any(r.max_steps % self.chunk for r in solves):
            raise ValueError("max_steps must be a multiple of the chunk")
        tol, max_steps = (solves[0].tol, solves[0].max_steps) if solves else (0.0, 1)
        pending = sorted(requests, key=lambda r: r.arrival)
        queue = []
        imag = {}          # batch index -> [request, psi, last E, steps]
        retired = []       # batch indices of solves finished since the last rebind
        real = {}          # session -> (request, completion event)
        used = 0.0
        batch = Batch([], self.dtype)
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0  # noqa: E731
        while pending or queue or imag or real:
            now = clock()
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            # admission in arrival order: the memory budget and the device's free memory
            # for solves, a free session for segments
            changed = False
            keep = []
            free = self.mem_info()[0] - self.reserve if queue else 0
            short = None   # a solve the device's free memory could not take this round
            held = False   # ordered admission: an earlier request could not start
            for r in queue:
                if held:
                    keep.append(r)
                    continue
                running = len(imag) + len(real) if self.ordered else len(imag)
                full = self.max_active is not None and running >= self.max_active
                if r.kind == "imaginary":
                    need = state_bytes(r.inst.n, self.dtype)
                    if used + need > self.budget or full:
                        keep.append(r)
                        held = self.ordered
                        continue
                    if need > free:
                        self.refused += 1
                        short = short or (r, need)
                        keep.append(r)
                        held = self.ordered
                        continue
                    free -= need
                    with torch.cuda.stream(self.batch_stream):
                        idx = batch.add(r.inst)
                        psi = initial_states([r.inst], self.dtype, seed0=10_000 + r.rid)[0]
                    imag[idx] = [r, psi, float("nan"), 0]
                    used += need
                    changed = True
                else:
                    sess = self.sessions[r.session]
                    if sess.busy or (self.ordered and full):
                        keep.append(r)
                        held = self.ordered and not sess.busy
                        continue
                    sess.busy = True
                    st = self.streams[r.session]
                    with torch.cuda.stream(st):
                        sess.plan.step(sess.psi, r.steps, sess.step)   # whole segment, asynchronous
                        ev = torch.cuda.Event()
                        ev.record(st)
                    sess.step += r.steps
                    real[r.session] = (r, ev)
            queue = keep
            if short and not imag and not real:
                # nothing of ours is running to free memory: waiting would not end
                r, need = short
                raise MemoryError(f"request {r.rid} needs {need} bytes of device memory; the device has "
                                  f"{max(free, 0)} free beyond the {self.reserve}-byte reserve")
            if imag:
                with torch.cuda.stream(self.batch_stream):
                    if changed:
                        # one rebind for the admissions and every retirement since the
                        # last one (retired solves stayed bound, frozen, in between)
                        psis = [None] * len(batch.instances)
                        act = np.zeros(len(batch.instances), np.int32)
                        for idx, rec in imag.items():
                            psis[idx] = rec[1]
                            act[idx] = 1
                        batch.bind(psis, act)
                        for idx in retired:
                            batch.remove(idx)      # unbound now: leaves without a rebuild
                        retired.clear()
                    slots = len(batch.instances)
                    live = np.zeros(slots, np.int32)
                    steps = np.zeros(slots, np.int64)
                    e_last = np.full(slots, np.nan)
                    for idx, rec in imag.items():
                        live[idx], steps[idx], e_last[idx] = 1, rec[3], rec[2]
                    # checks on the device (first check of a solve: E_last NaN, no
                    # convergence); synchronises the batch stream only
                    diag = batch.run(self.chunk, self.checks_per_round, tol, max_steps, live, steps, e_last)
                now = clock()
                for idx in list(imag):
                    rec = imag[idx]
                    r = rec[0]
                    rec[2], rec[3] = float(e_last[idx]), int(steps[idx])
                    if not live[idx]:
                        r.done_at, r.taken = now, rec[3]
                        r.result = dict(N=diag[idx, 0], E=diag[idx, 4], mu=diag[idx, 5], psi=rec[1])
                        used -= state_bytes(r.inst.n, self.dtype)
                        del imag[idx]
                        retired.append(idx)
                # retired solves stay bound but frozen (their launches return at once)
                # until the next admission rebinds the batch
            elif real or queue:
                time.sleep(2e-4)
            elif pending:
                time.sleep(max(0.0, min(2e-3, pending[0].arrival - clock())))
            for s_ in list(real):
                r, ev = real[s_]
                if ev.query():
                    sess = self.sessions[s_]
                    r.done_at, r.taken = clock(), r.steps
                    with torch.cuda.stream(self.streams[s_]):
                        r.result = dict(N=sess.plan.norm(sess.psi), step=sess.step)
                    sess.busy = False
                    del real[s_]
        torch.cuda.synchronize()
        batch.close()
        return requests


def run_plain(requests, sessions, dtype=torch.complex64, chunk=20):
    """The same requests one at a time, in arrival order, through single plans, against
    the wall clock (a request starts when it has arrived and the previous one is done)."""
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: q.arrival):
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        if r.kind == "imaginary":
            inst = r.inst
            plan = Plan(inst.n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                        static_expr=inst.static_expr)
            psi = initial_states([inst], dtype, seed0=10_000 + r.rid)[0]
            last, steps = float("nan"), 0
            while True:
                plan.step(psi, chunk)
                steps += chunk
                d = plan.diagnostics(psi)
                conv = abs(d["E"] - last) / (chunk * abs(d["E"])) < r.tol
                last = d["E"]
                if conv or steps >= r.max_steps:
                    break
            r.taken = steps
            r.result = dict(N=d["N"], E=d["E"], mu=d["mu"], psi=psi)
            plan.close()
        else:
            sess = sessions[r.session]
            sess.plan.step(sess.psi, r.steps, sess.step)
            sess.step += r.steps
            r.taken = r.steps
            r.result = dict(N=sess.plan.norm(sess.psi), step=sess.step)
        torch.cuda.synchronize()
        r.done_at = time.perf_counter() - t0
    return requests


def fifo_summary(requests, service_s):
    """Latencies and throughput of serving ``requests`` one at a time in arrival
    order when request ``r`` takes ``service_s(r)`` seconds alone (a request
    starts when it has arrived and the previous one is done)."""
    done, lat, first = 0.0, [], None
    for r in sorted(requests, key=lambda q: q.arrival):
        first = r.arrival if first is None else first
        done = max(done, r.arrival) + service_s(r)
        lat.append(done - r.arrival)
    lat = np.array(lat)
    span = done - first
    return dict(requests=len(lat), solves_per_s=len(lat) / span, makespan_s=span,
                p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3))


def plan_service_costs(requests, sessions, dtype=torch.complex64, chunk=20, reps=5):
    """Seconds that ``run_plain`` spends on one request of each kind and size, by
    parts: an imaginary-time solve's set-up (plan, initial state, release) and
    each ``chunk`` steps with their energy check; a real-time segment's seconds
    per step (one multi-step call) and its closing norm.  Measured on this GPU."""
    imag = {}
    for n in sorted({r.inst.n for r in requests if r.kind == "imaginary"}):
        inst = next(r.inst for r in requests if r.kind == "imaginary" and r.inst.n == n)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            plan = Plan(inst.n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                        static_expr=inst.static_expr)
            psi = initial_states([inst], dtype, seed0=1)[0]
            plan.close()
        torch.cuda.synchronize()
        setup = (time.perf_counter() - t0) / reps
        plan = Plan(inst.n, inst.x, inst.k, dtype=dtype, kind="imaginary", beta=inst.beta, dt=inst.dt,
                    static_expr=inst.static_expr)
        plan.step(psi, chunk)
        plan.diagnostics(psi)
        t0 = time.perf_counter()
        for _ in range(reps):
            plan.step(psi, chunk)
            plan.diagnostics(psi)
        per_chunk = (time.perf_counter() - t0) / reps
        plan.close()
        imag[n] = (setup, per_chunk)
    real = {}
    for s_, sess in enumerate(sessions):
        psi = sess.psi.clone()
        sess.plan.step(psi, 10, 0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sess.plan.step(psi, 200, 10)
        torch.cuda.synchronize()
        per_step = (time.perf_counter() - t0) / 200
        t0 = time.perf_counter()
        sess.plan.norm(psi)
        real[s_] = (per_step, time.perf_counter() - t0)
    return imag, real


def summarise(requests):
    lat = np.array([r.done_at - r.arrival for r in requests])
    span = max(r.done_at for r in requests) - min(r.arrival for r in requests)
    return dict(requests=len(requests), solves_per_s=len(requests) / span, makespan_s=span,
                p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3))
