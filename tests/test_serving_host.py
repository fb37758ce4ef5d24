"""Host-side serving logic (no GPU): admission by footprint, slot limit, arrival order, error propagation,
latency summary and the synthetic request stream."""
import threading
import time

import numpy as np
import pytest

from graphgp_b200 import serving as sv


def _reqs(sizes, arrivals=None):
    arrivals = arrivals or [0.0] * len(sizes)
    return [sv.Request(i, "generate", np.zeros((n, 2), np.float32), 8, 8, np.zeros(2), np.zeros(2), None, a)
            for i, (n, a) in enumerate(zip(sizes, arrivals))]


class _Probe:
    def __init__(self, delay=0.01):
        self.lock = threading.Lock()
        self.in_use = 0
        self.in_flight = 0
        self.max_in_use = 0
        self.max_in_flight = 0
        self.delay = delay
        self.log = []

    def process(self, r, slot):
        with self.lock:
            self.in_use += r.n
            self.in_flight += 1
            self.max_in_use = max(self.max_in_use, self.in_use)
            self.max_in_flight = max(self.max_in_flight, self.in_flight)
            self.log.append((r.rid, self.in_flight))
        time.sleep(self.delay)
        with self.lock:
            self.in_use -= r.n
            self.in_flight -= 1
        return r.n * 2, {"slot": slot}


def test_budget_and_slots_respected():
    rng = np.random.default_rng(0)
    sizes = [int(x) for x in rng.integers(10, 100, 60)]
    pr = _Probe()
    sch = sv.Scheduler(slots=4, budget=200, footprint=lambda r: r.n, process=pr.process, slot_init=lambda: "s")
    res, wall = sch.run(_reqs(sizes), realtime=False)
    assert [r.rid for r in res] == list(range(60))
    assert all(r.output == 2 * r.n for r in res)
    assert pr.max_in_use <= 200 and sch.peak_in_use <= 200
    assert pr.max_in_flight <= 4 and sch.peak_in_flight <= 4
    assert sch.peak_in_flight >= 2  # work overlaps
    assert sch.admission_order == list(range(60))  # strict arrival order, no overtaking


def test_oversize_request_runs_alone():
    pr = _Probe()
    sch = sv.Scheduler(slots=4, budget=100, footprint=lambda r: r.n, process=pr.process)
    res, _ = sch.run(_reqs([30, 30, 500, 30, 30]), realtime=False)
    assert len(res) == 5
    big = [f for rid, f in pr.log if rid == 2]
    assert big == [1]  # admitted only when nothing else was in flight
    assert sch.admission_order == [0, 1, 2, 3, 4]


def test_large_head_blocks_smaller_followers():
    """Admission is in arrival order: a request that does not fit yet is not overtaken by smaller ones."""
    pr = _Probe(delay=0.02)
    sch = sv.Scheduler(slots=8, budget=100, footprint=lambda r: r.n, process=pr.process)
    sch.run(_reqs([60, 60, 10, 10]), realtime=False)
    order = [rid for rid, _ in pr.log]
    assert order.index(1) < order.index(2) < order.index(3)


def test_realtime_arrivals_and_latency():
    pr = _Probe(delay=0.005)
    arr = [0.0, 0.02, 0.04, 0.06]
    sch = sv.Scheduler(slots=2, budget=1 << 30, footprint=lambda r: r.n, process=pr.process)
    res, wall = sch.run(_reqs([10] * 4, arr), realtime=True)
    for r in res:
        assert r.start >= r.arrival - 1e-3
        assert r.end >= r.start and r.latency >= 0.004
    s = sv.summarize(res, wall)
    assert s["requests"] == 4 and s["p50_ms"] <= s["p99_ms"]
    assert wall >= 0.06


def test_error_propagates():
    def bad(r, slot):
        if r.rid == 3:
            raise RuntimeError("boom")
        return 0, {}

    sch = sv.Scheduler(slots=3, budget=1 << 30, footprint=lambda r: 1, process=bad)
    with pytest.raises(RuntimeError, match="boom"):
        sch.run(_reqs([5] * 10), realtime=False)


def test_slot_init_failure_propagates():
    def init():
        raise OSError("no stream")

    sch = sv.Scheduler(slots=2, budget=10, footprint=lambda r: 1, process=lambda r, s: (0, {}), slot_init=init)
    with pytest.raises(OSError):
        sch.run(_reqs([5] * 3), realtime=False)


def test_synthetic_stream_distribution():
    reqs = sv.synthetic_stream(n_requests=400, rate=2000.0, seed=3, median_n=2000, n_min=1000, n_max=20000,
                               n_bins=50)
    ns = np.array([r.n for r in reqs])
    assert ns.min() >= 1000 and ns.max() <= 20000
    for r in reqs:
        assert r.points.shape[1] in (2, 3) and r.points.dtype == np.float32
        assert r.k in (8, 16, 32) and r.n0 == max(r.k, min(256, r.n // 100))
        assert len(r.bins) == 50 and r.bins[0] == 0.0
        assert (r.payload is None) == (r.op == "logdet")
    ops = [r.op for r in reqs]
    assert 0.6 < ops.count("generate") / 400 < 0.8
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0)
    assert 0.1 < arr[-1] < 0.3  # 400 arrivals at 2000/s
