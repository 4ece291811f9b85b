"""Benchmark: split-step Strang steps/s of the real-time stirred 256^3 complex64 solve.

One "step" is one Strang step of the hot path (local half-step, 3-D FFT,
kinetic phase, inverse 3-D FFT, local half-step) over the whole 256^3 grid.

Workload ("large single solve", 256^3 complex64): trap V = (x^2 + 1.44 y^2 +
2.25 z^2)/2, box [-12,12)^3, g = 2000, dt = 2.5e-4 (oscillator units), rotating
Gaussian beam A = 10, w = 0.5, R = 2, angular rate ramped 0 -> 0.5 over the first
200 steps.  The plan runs in the reference's units (V x2, g x2, dt /2), which is
an exact reparametrisation.  Inputs are synthetic (seeded noisy Gaussian relaxed
for 50 imaginary-time steps); psi is 128 MiB, larger than the 126 MB L2.

On one GPU the line also carries ``plain_floor`` (the reference's step sequence
with cuFFT through torch.fft and byte-equivalent elementwise kernels: a floor on
the reference's step time on the same GPU, since its CuPy code cannot run here),
``stir512`` (the same physics at 512^3), ``batched`` (64 imaginary-time solves of mixed
grid sizes as one running batch vs one at a time: solves/s) and ``serving`` (a
seeded request stream through the continuous-batching server vs the plain path:
solves/s, p50/p99 latency, results identical) -- the other two parts of the
metric.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``
prints one JSON line (rank 0).  Multi-GPU runs are independent replicas (one
solve per GPU, weak scaling); ``value`` is the whole-job steps/s.
"""

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_GRID, L_BOX, G, DT = 256, 24.0, 2000.0, 2.5e-4
BEAM = dict(amp=10.0, width=0.5, radius=2.0, omega=0.5, ramp_steps=200)
TRAP_REF = "x**2+1.44*y**2+2.25*z**2"
METRIC = "steps/s & HBM roofline % at 256^3 c64"
WORKLOAD = ("stir256_c64: real-time stirred GPE, 256^3 complex64, box [-12,12)^3, g=2000, "
            "dt=2.5e-4, beam A=10 w=0.5 R=2 Omega 0->0.5 over 200 steps")
FALLBACK_HBM = 6650.0
# the sweep kernel of each axis in one real-time step at n = 256
KERNELS = {"z": "k_fast_occ<256, 0, float, 3, 3> (fused z sweep)",
           "y": "k_fast_occ<256, 1, float, 0, 4> (y sweep, 2 per step)",
           "x": "k_fast_occ<256, 2, float, 4, 3> (x sweep with kinetic phase)"}
TRAFFIC_KEYS = {"z": "sweep_z", "y": "sweep_y", "x": "sweep_x"}
# opt-in sweep paths (identical results): the kernels that replace the default ones
PATH_KERNELS = {"tma": {"y": ("k_tma_plain<256, 1> (TMA-staged y sweep, 2 per step)", "sweep_y_tma")},
                "plane": {"z": ("k_plane<256, float, 3> (inverse y, Z21, forward y per x-plane)", "plane")}}


def workload_config(world, path="default"):
    """The ``config`` of both arms' lines (the sweep path only when not the default)."""
    cfg = {"workload": WORKLOAD, "grid": N_GRID, "psi_bytes": N_GRID ** 3 * 8,
           "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
           "l2": "inputs larger than L2 (128 MiB psi vs 126 MB L2), no flush"}
    if path != "default":
        cfg["sweep_path"] = path
    return cfg


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM, "fallback"


# ------------------------------------------------------------------ distributed
def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if os.environ.get("GPE_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(value, world, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(ms, steps, world, device=None):
    """Whole-job steps/s of `world` replicas that each ran `steps` steps: the
    slowest rank's device time sets the job time.  Returns (max ms, steps/s)."""
    ms_max = max_over_ranks(ms, world, device)
    return ms_max, world * steps / (ms_max / 1e3)


def barrier(world, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """``nvidia-smi`` clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ workload
def grids():
    x = np.linspace(-L_BOX / 2, L_BOX / 2, N_GRID, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(N_GRID, L_BOX / N_GRID)
    return x, k


def initial_state(x, seed=0):
    """Seeded noisy Gaussian, normalised (host, complex128)."""
    n = len(x)
    rng = np.random.default_rng(seed)
    g = np.exp(-x ** 2 / 2)
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).astype(np.complex128)
    psi *= 1 + 0.01 * (rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))) / np.sqrt(2)
    dx = x[1] - x[0]
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * dx ** 3)
    return psi


def ours(args, world, rank, local):
    import torch
    from gpe_simulator_b200 import beam_in_reference_units, build
    from gpe_simulator_b200.plan import Plan, launch_count, profile, profile_read
    build.build()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    x, k = grids()
    beam = beam_in_reference_units(BEAM["amp"], BEAM["width"], BEAM["radius"], BEAM["omega"],
                                   BEAM["ramp_steps"] * DT)
    plan = Plan(N_GRID, x, k, dtype=torch.complex64, kind="real", beta=2 * G, dt=DT / 2,
                static_expr=TRAP_REF, beam=beam, path=args.path)
    args.path = plan.path   # "auto" resolved
    prep = Plan(N_GRID, x, k, dtype=torch.complex64, kind="imaginary", beta=2 * G, dt=DT,
                static_expr=TRAP_REF)
    host0 = initial_state(x, seed=rank).astype(np.complex64)
    psi = torch.from_numpy(host0).to(device)
    prep.step(psi, 50)
    plan.step(psi, args.warmup, 0)
    torch.cuda.synchronize()

    # ---- timed region: K steps, one multi-step C-ABI call, inputs resident in HBM
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.6)
    n0 = launch_count(plan)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world, device)
    torch.cuda.synchronize()
    start.record()
    plan.step(psi, args.steps, args.warmup)
    end.record()
    torch.cuda.synchronize()
    barrier(world, device)
    launches = launch_count(plan) - n0
    ms = start.elapsed_time(end)
    clocks = sampler.stop()
    ms_max, value = job_throughput(ms, args.steps, world, device)

    # ---- per-launch durations of the sweeps (events around each launch, same stream)
    profile(plan, True)
    plan.step(psi, args.steps, args.warmup + args.steps)
    per = profile_read(plan)
    profile(plan, False)
    torch.cuda.synchronize()
    dom = max(per, key=lambda a: per[a][0])
    dom_ms, dom_n = per[dom]
    s_bytes = 8
    m = N_GRID ** 3
    bytes_per_launch = 2 * s_bytes * m
    achieved = bytes_per_launch / (dom_ms / dom_n / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    kernel, tkey = KERNELS[dom], TRAFFIC_KEYS[dom]
    if dom in PATH_KERNELS.get(args.path, {}):
        kernel, tkey = PATH_KERNELS[args.path][dom]
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(tkey)

    # ---- end to end: public closure API with host buffers, H2D + D2H every step
    from gpe_simulator_b200.make_propagator import make_real_propagator
    from types import SimpleNamespace
    from gpe_simulator_b200.expressions import cuda_expression
    st = SimpleNamespace(
        type="real", N_grids=N_GRID, beta=2 * G, dt=DT / 2, beam=beam, kinetic_coeff=1.0,
        x_array=torch.from_numpy(x).to(device), k_array=torch.from_numpy(k).to(device),
        staticV=torch.zeros((N_GRID,) * 3, dtype=torch.complex128, device=device),
        potential_params=dict(static=dict(activate=True, expression=cuda_expression(TRAP_REF)),
                              dynamic=dict(activate=False, expression="0")),
        k_cut_params=dict(activate=False, k_cut=0.0), psi=psi)
    prop = make_real_propagator(st)
    host = torch.from_numpy(host0).pin_memory()
    outs = [torch.empty_like(host).pin_memory() for _ in range(2)]
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    prop(st, 0.0)
    # Every step copies its input from pinned host memory, runs the closure and
    # copies its result back.  Two device buffers and one stream per engine
    # (upload, compute, download) let step i's upload and step i-1's download
    # overlap step i's neighbours, as a streaming caller would run them.
    bufs = [psi, torch.empty_like(psi)]
    s_up, s_run, s_down = torch.cuda.Stream(device), torch.cuda.Stream(device), torch.cuda.Stream(device)
    up_done = [torch.cuda.Event() for _ in range(2)]
    run_done = [torch.cuda.Event() for _ in range(2)]
    down_done = [torch.cuda.Event() for _ in range(2)]
    torch.cuda.synchronize()
    barrier(world, device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_up)
    for i in range(e2e_steps):
        b = i % 2
        if i >= 2:
            s_up.wait_event(down_done[b])          # buffer b's previous result has left
        with torch.cuda.stream(s_up):
            bufs[b].copy_(host, non_blocking=True)
            up_done[b].record(s_up)
        s_run.wait_event(up_done[b])
        with torch.cuda.stream(s_run):
            st.psi = bufs[b]
            prop(st, (args.warmup + i) * st.dt)
            run_done[b].record(s_run)
        s_down.wait_event(run_done[b])
        with torch.cuda.stream(s_down):
            outs[b].copy_(bufs[b], non_blocking=True)
            down_done[b].record(s_down)
    cur = torch.cuda.current_stream(device)
    for ev in down_done:
        cur.wait_event(ev)
    e1.record(cur)
    torch.cuda.synchronize()
    st.psi = psi
    e2e_ms, e2e = job_throughput(e0.elapsed_time(e1), e2e_steps, world, device)
    nbytes = host.numel() * host.element_size()

    result = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded noisy Gaussian relaxed 50 imaginary steps)",
        "config": workload_config(world, args.path),
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                     "traffic_source": "profiles/traffic.json (ncu dram bytes read + write per launch)",
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "avg_launch_ms": dom_ms / dom_n,
                     "per_axis_ms": {a: per[a][0] / max(per[a][1], 1) for a in per}},
        "step_roofline": {"algorithmic_bytes_per_step": 6 * s_bytes * m,
                          "achieved_gbs": 6 * s_bytes * m * value / world / 1e9,
                          "frac": 6 * s_bytes * m * value / world / 1e9 / peak},
        "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "steps": e2e_steps,
                "path": "make_real_propagator closure per step, psi H2D from pinned host before "
                        "and D2H after every step; upload, compute and download on separate "
                        "streams with two device buffers (copies of neighbouring steps overlap)"},
        "clocks": clocks,
    }
    if world == 1 and rank == 0 and not args.no_cpu:
        result["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    if world == 1 and not args.no_plain:
        result["plain_floor"] = plain_floor_leg()
    if world == 1 and not args.no_large:
        result["stir512"] = large_leg()
    if world == 1 and not args.no_expr:
        result["expression_beam"] = expression_leg()
    if world == 1 and not args.no_batch:
        result["batched"] = batched_leg()
    if world == 1 and not args.no_serve:
        result["serving"] = serving_leg(args.serve_requests, args.serve_rates, args.serve_measure_one_at_a_time)
    return result, plan


def expression_leg(steps=200, warmup=5):
    """The stirring beam written in the reference's expression grammar (the form a
    YAML stage carries, ``gpe/make_kernel.py:14-45``) against the built-in beam,
    256^3 complex64, same state: steps/s of one multi-step call and of per-step
    ``make_real_propagator`` closure calls, state resident, and the relative
    difference of the two final states."""
    import torch
    from types import SimpleNamespace
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    from gpe_simulator_b200.expressions import cuda_expression
    from gpe_simulator_b200.make_propagator import make_real_propagator
    from gpe_simulator_b200.plan import launch_count
    x, k = grids()
    beam = beam_in_reference_units(BEAM["amp"], BEAM["width"], BEAM["radius"], BEAM["omega"],
                                   BEAM["ramp_steps"] * DT)
    expr = beam.expression()
    g = torch.from_numpy(np.exp(-x ** 2 / 2)).cuda()
    base = (g[:, None, None] * g[None, :, None] * g[None, None, :]).to(torch.complex64).contiguous()
    out = {"expression": expr}
    finals = {}
    for name, kw in (("builtin", dict(beam=beam)), ("expression", dict(dynamic_expr=expr))):
        plan = Plan(N_GRID, x, k, dtype=torch.complex64, kind="real", beta=2 * G, dt=DT / 2,
                    static_expr=TRAP_REF, **kw)
        psi = base.clone()
        plan.normalise(psi)
        plan.step(psi, warmup, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        n0 = launch_count(plan)
        e0.record()
        plan.step(psi, steps, warmup)
        e1.record()
        torch.cuda.synchronize()
        out[f"{name}_steps_per_s"] = steps * 1e3 / e0.elapsed_time(e1)
        out[f"{name}_launches_per_step"] = (launch_count(plan) - n0) / steps
        finals[name] = psi
        plan.close()
        # the drop-in closure, one call per step (as gpe/launch.py:8-13 calls it)
        pp = dict(static=dict(activate=True, expression=cuda_expression(TRAP_REF)),
                  dynamic=dict(activate=name == "expression",
                               expression=cuda_expression(expr, True) if name == "expression" else "0"))
        st = SimpleNamespace(type="real", N_grids=N_GRID, beta=2 * G, dt=DT / 2, kinetic_coeff=1.0,
                             beam=beam if name == "builtin" else None,
                             x_array=torch.from_numpy(x).cuda(), k_array=torch.from_numpy(k).cuda(),
                             staticV=torch.zeros((N_GRID,) * 3, dtype=torch.complex128, device="cuda"),
                             potential_params=pp, k_cut_params=dict(activate=False, k_cut=0.0),
                             psi=base.clone())
        prop = make_real_propagator(st)
        for i in range(warmup):
            prop(st, i * st.dt)
        torch.cuda.synchronize()
        e0.record()
        for i in range(steps):
            prop(st, (warmup + i) * st.dt)
        e1.record()
        torch.cuda.synchronize()
        out[f"{name}_closure_steps_per_s"] = steps * 1e3 / e0.elapsed_time(e1)
        del st, prop
    d = finals["expression"].to(torch.complex128) - finals["builtin"].to(torch.complex128)
    out["rel_diff_final_psi"] = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(
        finals["builtin"].to(torch.complex128)))
    out["ratio_multistep"] = out["expression_steps_per_s"] / out["builtin_steps_per_s"]
    out["ratio_closure"] = out["expression_closure_steps_per_s"] / out["builtin_closure_steps_per_s"]
    out["steps"] = steps
    torch.cuda.empty_cache()
    return out


def large_leg(steps=100, warmup=5):
    """The 512^3 complex64 single solve (same trap, beam, g and dt as the 256^3
    workload, box [-12,12)^3): steps/s of one multi-step call, state resident."""
    import torch
    from gpe_simulator_b200 import Plan, beam_in_reference_units
    n = 512
    x = np.linspace(-L_BOX / 2, L_BOX / 2, n, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(n, L_BOX / n)
    beam = beam_in_reference_units(BEAM["amp"], BEAM["width"], BEAM["radius"], BEAM["omega"],
                                   BEAM["ramp_steps"] * DT)
    plan = Plan(n, x, k, dtype=torch.complex64, kind="real", beta=2 * G, dt=DT / 2, static_expr=TRAP_REF,
                beam=beam)
    g = torch.from_numpy(np.exp(-x ** 2 / 2)).cuda()
    psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).to(torch.complex64).contiguous()
    plan.normalise(psi)
    plan.step(psi, warmup, 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    plan.step(psi, steps, warmup)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    m = n ** 3
    plan.close()
    del psi
    torch.cuda.empty_cache()
    peak, _ = measured_peak()
    return {"grid": n, "steps": steps, "steps_per_s": 1e3 / ms, "ms_per_step": ms,
            "step_roofline_frac": 6 * 8 * m / (ms / 1e3) / 1e9 / peak,
            "data": "Gaussian trap state, synthetic"}


def plain_floor_leg(steps=50, warmup=5):
    """Floor of the reference's own step time on this GPU (CuPy is not installed,
    so its code cannot run here): the reference's sequence per step -- half-step
    kernel, fftn, kinetic kernel, ifftn, half-step kernel -- with cuFFT through
    torch.fft (out of place, as cp.fft) and each elementwise RawKernel replaced
    by one torch kernel moving the same bytes (half-step: psi and staticV read,
    psi written, 48 B/point in complex128; kinetic: psi_k read and written) but
    doing less arithmetic.  complex128 as the reference ships, complex64 for
    comparison; the reference's steps cannot be faster than these."""
    import torch
    out = {}
    n = N_GRID
    for name, dtype in (("c128", torch.complex128), ("c64", torch.complex64)):
        g = torch.Generator(device="cuda").manual_seed(0)
        real = torch.float64 if dtype == torch.complex128 else torch.float32
        psi = torch.randn((n, n, n), dtype=dtype, device="cuda", generator=g)
        # unit-modulus factors keep repeated steps finite and normal
        ang = torch.randn((n, n, n), dtype=real, device="cuda", generator=g)
        pot = torch.polar(torch.ones_like(ang), ang)
        del ang

        def step(psi):
            torch.mul(psi, pot, out=psi)
            f = torch.fft.fftn(psi)
            f.mul_(complex(0.6, 0.8))
            psi = torch.fft.ifftn(f)
            torch.mul(psi, pot, out=psi)
            return psi

        for _ in range(warmup):
            psi = step(psi)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            psi = step(psi)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_step": ms, "steps_per_s": 1e3 / ms}
        del psi, pot
        torch.cuda.empty_cache()
    out["note"] = ("reference step sequence at 256^3: cuFFT via torch.fft + byte-equivalent torch "
                   "elementwise kernels in place of its RawKernels; a floor on its step time")
    return out


def plain_form_costs(n, dtype, real_time=False, steps=100, checks=10):
    """Device milliseconds per step and per energy check of the reference's plain
    form on this GPU (CuPy is not installed here, so its own code cannot run):
    per step, looped from Python as ``gpe/launch.py:8-13`` loops, the kernel
    sequence of ``gpe/make_propagator.py:109-151`` (``57-103`` in real time) --
    half-step, ``fftn``, kinetic factor, ``ifftn``, half-step, and in imaginary
    time the two-pass norm and the division of ``gpe/helper.py:81-93``; per
    check, the ``fftn`` of the state and the E_kin, E_pot, E_int sums read on the
    host (the convergence rule).  cuFFT runs through torch.fft; each elementwise
    RawKernel is one torch kernel moving the same bytes (the half-step reads psi
    and its potential array and writes psi), so the reference's own steps cannot
    be faster.  Times include the gaps of the Python loop."""
    import torch
    real = torch.float64 if dtype == torch.complex128 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(n)
    psi = torch.randn((n, n, n), dtype=dtype, device="cuda", generator=g)
    psi /= torch.linalg.vector_norm(psi)
    # the half-step's potential array (float64 in imaginary time, complex128 U - iGamma in
    # real time) and a unit-modulus stand-in factor for the arithmetic
    if real_time:
        pot = torch.polar(torch.ones((n, n, n), dtype=real, device="cuda"),
                          torch.randn((n, n, n), dtype=real, device="cuda", generator=g))
    else:
        pot = torch.ones((n, n, n), dtype=real, device="cuda")
    k2 = torch.rand((n, n, n), dtype=real, device="cuda", generator=g)

    def step(psi):
        torch.mul(psi, pot, out=psi)
        f = torch.fft.fftn(psi)
        f.mul_(complex(0.6, 0.8))
        psi = torch.fft.ifftn(f)
        torch.mul(psi, pot, out=psi)
        if not real_time:
            psi.div_(torch.linalg.vector_norm(psi))
        return psi

    def check(psi):
        f = torch.fft.fftn(psi)
        e_kin = (f.abs().square() * k2).sum()
        rho = psi.abs().square()
        return float(e_kin + (rho * k2).sum() + rho.square().sum())   # host read, as the rule needs

    for _ in range(3):
        psi = step(psi)
    check(psi)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        psi = step(psi)
    e1.record()
    torch.cuda.synchronize()
    per_step = e0.elapsed_time(e1) / steps
    e0.record()
    for _ in range(checks):
        check(psi)
    e1.record()
    torch.cuda.synchronize()
    per_check = e0.elapsed_time(e1) / checks
    del psi, pot, k2
    return per_step, per_check


PLAIN_FORM_NOTE = ("the reference's per-step sequence looped from Python (cuFFT via torch.fft, byte-equivalent "
                   "elementwise kernels, normalise every imaginary step, an energy check every 10 (batched) or "
                   "20 (served) steps): device ms per step and per check measured per grid size, times each "
                   "solve's step count; c128 as the reference ships, c64 for comparison")


def batched_leg():
    """Batched parameter sweep: 64 imaginary-time solves (grids 48^3..160^3, g
    log-uniform in [100, 5000], trap aspect ratios in [0.5, 2], complex64, dt =
    1e-3 in oscillator units) run to |dE|/E < 1e-9 per step or 5000 steps, as one
    running batch and one at a time through single plans with the same
    convergence checks (every 10 steps).  Wall-clock seconds, states resident."""
    import torch
    from gpe_simulator_b200.batch import Batch, initial_states, solve_alone, sweep_instances
    insts = sweep_instances(64, seed=1)
    states = initial_states(insts, torch.complex64)
    batch = Batch(insts, torch.complex64)
    work = [st.clone() for st in states]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps, final = batch.solve(work, tol=1e-9, max_steps=5000, check_every=10)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    launches = batch.launch_count()
    batch.close()
    t0 = time.perf_counter()
    alone = []
    for inst, st in zip(insts, states):
        alone.append(solve_alone(inst, st.clone(), torch.complex64, tol=1e-9, max_steps=5000, check_every=10))
    torch.cuda.synchronize()
    t_alone = time.perf_counter() - t0
    a_steps = np.array([a[0] for a in alone])
    a_diag = np.array([a[1] for a in alone])
    e_diff = float(np.max(np.abs(final[:, 4] - a_diag[:, 4]) / np.abs(a_diag[:, 4])))
    # error against the FP64 run at the same dt for a sample (one instance per grid size):
    # the complex128 plan from the same start for the same number of steps
    from gpe_simulator_b200 import Plan
    psi_err = {}
    for n in sorted({i.n for i in insts}):
        i = next(j for j, inst in enumerate(insts) if inst.n == n)
        inst = insts[i]
        ref = Plan(inst.n, inst.x, inst.k, dtype=torch.complex128, kind="imaginary", beta=inst.beta, dt=inst.dt,
                   static_expr=inst.static_expr)
        b = states[i].to(torch.complex128).contiguous()
        ref.step(b, int(steps[i]))
        d = work[i].to(torch.complex128) - b
        psi_err[str(n)] = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(b))
        ref.close()
    # the reference's plain form, one solve at a time, each for the steps it needs
    plain = {}
    for name, dtype in (("c128", torch.complex128), ("c64", torch.complex64)):
        cost = {n: plain_form_costs(n, dtype) for n in sorted({i.n for i in insts})}
        ms = sum(int(k) * cost[inst.n][0] + (int(k) // 10) * cost[inst.n][1] for inst, k in zip(insts, steps))
        plain[name] = ms / 1e3
    torch.cuda.empty_cache()
    return {"instances": len(insts), "grids": sorted({i.n for i in insts}),
            "solves_per_s": len(insts) / t_batch, "wall_s": t_batch,
            "one_at_a_time_solves_per_s": len(insts) / t_alone, "one_at_a_time_wall_s": t_alone,
            "speedup": t_alone / t_batch,
            "plain_form_solves_per_s": {k: len(insts) / v for k, v in plain.items()},
            "speedup_vs_plain_form": {k: v / t_batch for k, v in plain.items()},
            "plain_form": PLAIN_FORM_NOTE,
            "psi_err_vs_fp64_same_dt": psi_err,
            "steps_median": int(np.median(steps)), "steps_max": int(steps.max()),
            "same_steps_as_alone": bool(np.array_equal(steps, a_steps)),
            "E_max_rel_diff_vs_alone": e_diff, "gpu_launches": int(launches),
            "criterion": "|E_k - E_{k-10}| / (10 |E_k|) < 1e-9 or 5000 steps"}


# requests running at once in the serving leg (solves and segments, admitted in
# arrival order): 8 kept the median near first come, first served; 4 lost
# throughput (6.13 vs 6.49 solves/s on the 1000-request stream)
SERVE_MAX_ACTIVE = 8


def serving_leg(count, rates, measure_one_at_a_time=False):
    """Serving stream (config 5): ``count`` requests with seeded Poisson arrivals at
    each rate of ``rates``; 70% imaginary-time ground states 32^3..128^3 and 30%
    real-time stirring segments of 500-5000 steps on 8 resident states
    64^3..256^3, complex64, 150 GB budget and the device's free memory, through
    the continuous-batching server (measured, wall clock).

    One request at a time on the same arrivals: a FIFO schedule over each
    request's service time alone, for this library's single plans (set-up, steps
    and checks at per-size costs measured here, times the request's step count)
    and for the reference's plain form (its per-step sequence, ``plain_form_costs``).
    With ``measure_one_at_a_time`` the single-plan path also runs the whole stream
    (``serve.run_plain``) and results are checked identical to the server's."""
    import torch
    from gpe_simulator_b200 import serve
    out = {"requests": count, "max_active_solves": SERVE_MAX_ACTIVE, "budget_bytes": 150e9, "rates": []}
    grids = [n for n, _ in serve.SESSION_GRIDS]
    for rate in rates:
        reqs = serve.workload(count, rate=rate, seed=2)
        sess = serve.make_sessions()
        srv = serve.Server(sess, budget=150e9, max_active=SERVE_MAX_ACTIVE)
        t0 = time.perf_counter()
        srv.run(reqs)
        wall = time.perf_counter() - t0
        mixed = serve.summarise(reqs)
        row = {"rate_per_s": rate, "imaginary": sum(r.kind == "imaginary" for r in reqs),
               "solves_per_s": mixed["solves_per_s"], "p50_ms": mixed["p50_ms"], "p99_ms": mixed["p99_ms"],
               "makespan_s": mixed["makespan_s"], "admissions_deferred_for_memory": srv.refused, "wall_s": wall}
        # one at a time through single plans: FIFO over measured per-size costs
        sess_model = serve.make_sessions(relax_steps=20)
        icost, rcost = serve.plan_service_costs(reqs, sess_model)

        def own(r):
            if r.kind == "imaginary":
                setup, per_chunk = icost[r.inst.n]
                return setup + (r.taken // 20) * per_chunk
            per_step, tail = rcost[r.session]
            return r.taken * per_step + tail

        mod = serve.fifo_summary(reqs, own)
        row.update({"one_at_a_time_solves_per_s": mod["solves_per_s"], "one_at_a_time_p50_ms": mod["p50_ms"],
                    "one_at_a_time_p99_ms": mod["p99_ms"], "speedup": mixed["solves_per_s"] / mod["solves_per_s"]})
        # the reference's plain form, one at a time, on the same arrivals
        for name, dtype in (("c128", torch.complex128), ("c64", torch.complex64)):
            icp = {n: plain_form_costs(n, dtype, steps=60, checks=6)
                   for n in sorted({r.inst.n for r in reqs if r.kind == "imaginary"})}
            rcp = {n: plain_form_costs(n, dtype, real_time=True, steps=60, checks=2) for n in sorted(set(grids))}

            def plain(r):
                if r.kind == "imaginary":
                    step, chk = icp[r.inst.n]
                    return (r.taken * step + (r.taken // 20) * chk) / 1e3
                step, chk = rcp[grids[r.session]]
                return (r.taken * step + chk) / 1e3

            pf = serve.fifo_summary(reqs, plain)
            row[f"plain_form_{name}"] = {"solves_per_s": pf["solves_per_s"], "p50_ms": pf["p50_ms"],
                                         "p99_ms": pf["p99_ms"]}
            row[f"speedup_vs_plain_form_{name}"] = mixed["solves_per_s"] / pf["solves_per_s"]
        torch.cuda.empty_cache()
        if measure_one_at_a_time:
            reqs2 = serve.workload(count, rate=rate, seed=2)
            sess2 = serve.make_sessions()
            serve.run_plain(reqs2, sess2)
            meas = serve.summarise(reqs2)
            same = all(a.taken == b.taken and (a.kind != "imaginary" or torch.equal(a.result["psi"], b.result["psi"]))
                       for a, b in zip(reqs, reqs2))
            same = same and all(torch.equal(x.psi, y.psi) for x, y in zip(sess, sess2))
            row["one_at_a_time_measured"] = {"solves_per_s": meas["solves_per_s"], "p50_ms": meas["p50_ms"],
                                             "p99_ms": meas["p99_ms"], "results_identical": bool(same)}
            for s_ in sess2:
                s_.plan.close()
        for s_ in sess + sess_model:
            s_.plan.close()
        out["rates"].append(row)
        torch.cuda.empty_cache()
    out["one_at_a_time"] = ("FIFO schedule on the same arrivals over each request's time alone: this "
                            "library's single plans at per-size costs measured here (plan set-up, 20-step "
                            "chunks with their energy check, per-step cost of each resident session) times "
                            "the request's steps")
    out["plain_form"] = PLAIN_FORM_NOTE
    out.update({k: out["rates"][0][k] for k in ("rate_per_s", "solves_per_s", "p50_ms", "p99_ms",
                                                 "one_at_a_time_solves_per_s", "one_at_a_time_p50_ms",
                                                 "one_at_a_time_p99_ms", "speedup",
                                                 "speedup_vs_plain_form_c128", "speedup_vs_plain_form_c64")})
    return out


def cpu_baseline(budget_s, steps_cap=None):
    """The oracle port (NumPy + scipy.fft, all host threads) on the same workload."""
    from oracle import ssf
    from oracle.ssf import Beam, Model
    x, _ = grids()
    b = Beam(2 * BEAM["amp"], BEAM["width"], BEAM["radius"], 2 * BEAM["omega"],
             BEAM["ramp_steps"] * DT / 2)
    model = Model(n=N_GRID, simulation_range=L_BOX, kind="real", beta=2 * G, dt=DT / 2,
                  static_expr=TRAP_REF, beam=b)
    psi = initial_state(x).astype(np.complex64)
    t0 = time.perf_counter()
    psi = ssf.step(psi, model, 0.0)
    one = time.perf_counter() - t0
    n = max(1, int(budget_s / max(one, 1e-3)))
    if steps_cap:
        n = min(n, steps_cap)
    t0 = time.perf_counter()
    for i in range(n):
        psi = ssf.step(psi, model, (i + 1) * model.dt)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "steps/s", "cores": ssf.WORKERS, "kind": "port",
            "sample": f"{n} Strang steps of the 256^3 workload in complex64 (oracle port, "
                      f"scipy.fft workers={ssf.WORKERS}) after 1 untimed step"}


def reference(args, world, rank):
    """The reference arm: the oracle port of the reference algorithm on host cores."""
    if rank != 0:
        return None
    budget = float(os.environ.get("GPE_REFERENCE_SECONDS", "60"))
    base = cpu_baseline(budget, steps_cap=args.steps)
    return {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic", "config": workload_config(world),
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--e2e-steps", type=int, default=40)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sweep leg")
    ap.add_argument("--no-large", action="store_true", help="skip the 512^3 leg")
    ap.add_argument("--no-expr", action="store_true",
                    help="skip the leg with the beam as a reference-grammar expression")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the floor of the reference's step sequence (cuFFT via torch.fft)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--path", choices=("default", "tma", "plane", "auto"), default="default",
                    help="sweep path of the main leg: default, tma (y/x pencils staged by TMA), "
                         "plane (y/z sweeps fused per x-plane), auto (timed once per device and "
                         "cached); identical results")
    ap.add_argument("--serve-requests", type=int, default=1000, help="requests of the serving stream")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[50.0],
                    help="Poisson arrival rates (requests/s) of the serving stream")
    ap.add_argument("--serve-measure-one-at-a-time", action="store_true",
                    help="also run the whole stream one request at a time through single plans")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
        out = reference(args, world, rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    world, rank, local = dist_init(args.gpus)
    out, plan = ours(args, world, rank, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    plan.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
