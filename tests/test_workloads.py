"""Host logic of the batched sweep and the serving stream (no GPU): the seeded
instance and request generators follow the stated distributions, and the
latency summary is the percentile of completion minus arrival."""

import math
import re

import numpy as np
import pytest

from gpe_simulator_b200 import batch, serve
from gpe_simulator_b200.expressions import split_static

TRAP = re.compile(r"x\*\*2\+(.+)\*y\*\*2\+(.+)\*z\*\*2")


def test_sweep_instances_follow_the_batched_configuration():
    insts = batch.sweep_instances(64, seed=1)
    assert len(insts) == 64
    again = batch.sweep_instances(64, seed=1)
    assert [(i.n, i.beta, i.static_expr) for i in insts] == [(i.n, i.beta, i.static_expr) for i in again]
    sizes = {48: 12.0, 64: 16.0, 96: 20.0, 128: 24.0, 160: 28.0}      # box [-L, L)
    for inst in insts:
        assert sizes[inst.n] == inst.simulation_range
        assert 200.0 <= inst.beta <= 10000.0                          # 2 g, g in [100, 5000]
        assert inst.dt == pytest.approx(5e-4)                         # oscillator 1e-3, halved
        ly2, lz2 = (float(v) for v in TRAP.fullmatch(inst.static_expr).groups())
        assert 0.25 <= ly2 <= 4.0 and 0.25 <= lz2 <= 4.0              # lambda in [0.5, 2]
        assert any(split_static(inst.static_expr))                    # a program the plan accepts
        np.testing.assert_allclose(inst.x[1] - inst.x[0], inst.simulation_range / inst.n)
        assert inst.k[1] == pytest.approx(2 * math.pi / inst.simulation_range)
    counts = {n: sum(i.n == n for i in insts) for n in sizes}
    assert counts == {48: 11, 64: 14, 96: 13, 128: 11, 160: 15}


def test_request_stream_follows_the_serving_configuration():
    reqs = serve.workload(count=1000, rate=20.0, seed=2)
    assert [r.rid for r in reqs] == list(range(1000))
    arrivals = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arrivals) > 0)
    assert arrivals[-1] / 1000 == pytest.approx(1 / 20.0, rel=0.1)     # Poisson at 20/s
    imag = [r for r in reqs if r.kind == "imaginary"]
    real = [r for r in reqs if r.kind == "real"]
    assert len(imag) + len(real) == 1000
    assert len(imag) / 1000 == pytest.approx(0.7, abs=0.04)
    assert {r.inst.n for r in imag} <= {32, 48, 64, 96, 128}
    assert all(200.0 <= r.inst.beta <= 10000.0 for r in imag)
    assert all(500 <= r.steps <= 5000 and 0 <= r.session < serve.SESSIONS for r in real)
    assert {n for n, _ in serve.SESSION_GRIDS} <= {64, 96, 128, 256}
    again = serve.workload(count=1000, rate=20.0, seed=2)
    assert [(r.kind, r.arrival) for r in again] == [(r.kind, r.arrival) for r in reqs]


def test_latency_summary():
    reqs = serve.workload(count=100, rate=50.0, seed=3)
    for i, r in enumerate(reqs):
        r.done_at = r.arrival + 0.01 * (i + 1)
    s = serve.summarise(reqs)
    lat = np.array([0.01 * (i + 1) for i in range(100)])
    assert s["requests"] == 100
    assert s["p50_ms"] == pytest.approx(np.percentile(lat, 50) * 1e3)
    assert s["p99_ms"] == pytest.approx(np.percentile(lat, 99) * 1e3)
    span = max(r.done_at for r in reqs) - min(r.arrival for r in reqs)
    assert s["solves_per_s"] == pytest.approx(100 / span)
