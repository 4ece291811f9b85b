"""Run-time choice of the sweep path (the autotuner of the register-resident sweeps).

For complex64 at n = 128 and 256, three sweep paths compute identical bits:

* ``"default"``: register-resident sweeps with plain loads;
* ``"tma"``: the y/x pencils staged by TMA in persistent launches;
* ``"plane"``: the y and z sweeps of each x-plane fused into one launch.

Which is fastest depends on the device, its clocks and how neighbouring
launches overlap, so :func:`choose_path` times a short multi-step call of each
candidate on a synthetic state of the plan's size and kind.  The winner is
cached per (device, n, dtype, kind) in a JSON file (``GPE_TUNE_CACHE``,
default ``~/.cache/gpe_simulator_b200/paths.json``) together with the measured
times.  Since the candidates produce identical results, the choice never
changes a solution.  Other sizes and complex128 have a single register-resident
path.  The FFT splits and lines per tile of each size are compiled in, chosen
from offline measurements.
"""

import json
import os
from pathlib import Path

import numpy as np
import torch

CANDIDATES = ("default", "tma", "plane")


def candidates(n, dtype):
    """Sweep paths available for grid size ``n`` and ``dtype``."""
    return CANDIDATES if dtype == torch.complex64 and int(n) in (128, 256) else ("default",)


def cache_path():
    return Path(os.environ.get("GPE_TUNE_CACHE", Path.home() / ".cache" / "gpe_simulator_b200" / "paths.json"))


def _load():
    try:
        return json.loads(cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(cache):
    path = cache_path()
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
    os.replace(tmp, path)


def _key(device_name, n, dtype, kind):
    return f"{device_name}|n={int(n)}|{str(dtype).replace('torch.', '')}|{kind}"


def time_path(n, x_array, k_array, dtype, kind, path, steps=20, reps=3):
    """Milliseconds per step of ``path``: the best of ``reps`` multi-step calls of
    ``steps`` steps on a Gaussian in a harmonic trap (CUDA events, current stream)."""
    from .plan import Plan
    x = np.asarray(x_array, dtype=np.float64)
    plan = Plan(n, x, k_array, dtype=dtype, kind=kind, beta=1000.0, dt=1e-4,
                static_expr="x**2+y**2+z**2", path=path)
    try:
        g = torch.from_numpy(np.exp(-x * x / 2)).cuda()
        psi = (g[:, None, None] * g[None, :, None] * g[None, None, :]).to(dtype).contiguous()
        plan.step(psi, 2, 0)
        best = float("inf")
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            plan.step(psi, steps, 2)
            b.record()
            b.synchronize()
            best = min(best, a.elapsed_time(b) / steps)
        return best
    finally:
        plan.close()


def choose_path(n, x_array, k_array, dtype, kind, device_name=None, timer=None):
    """The fastest sweep path for this (device, n, dtype, kind): from the cache, or
    timed now (``timer(path) -> ms per step``, default :func:`time_path`) and cached."""
    cands = candidates(n, dtype)
    if len(cands) == 1:
        return cands[0]
    if device_name is None:
        device_name = torch.cuda.get_device_name()
    key = _key(device_name, n, dtype, kind)
    cache = _load()
    hit = cache.get(key)
    if hit and hit.get("path") in cands:
        return hit["path"]
    if timer is None:
        timer = lambda p: time_path(n, x_array, k_array, dtype, kind, p)  # noqa: E731
    times = {p: float(timer(p)) for p in cands}
    best = min(times, key=times.get)
    cache[key] = {"path": best, "ms_per_step": times}
    _store(cache)
    return best
