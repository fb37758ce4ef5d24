"""Continuous-batching request loop for generate / inverse / log-determinant requests of uneven N, d and k.

Requests arrive over time (``Request.arrival`` seconds after the run starts). The engine keeps ``slots``
worker threads, each with its own CUDA stream; a request is admitted as soon as a slot is free and its
device-memory footprint fits in what the requests in flight leave of ``hbm_budget`` (admission is in arrival
order: a large request waits for memory rather than being overtaken). An admitted request uploads its
points, builds its graph on the device, runs its operation and copies the result back, all on its slot's
stream, so the device overlaps the work of every request in flight while the host thread of a slot only waits
on its own stream. A request that names a ``graph_key`` / ``table_key`` seen before reuses the graph / kernel
table that stays resident on the device.

Latency is completion time minus arrival time (queueing included); ``Engine.run`` returns the per-request
results and a summary with p50 / p99 latency, requests/s and points/s.

Note on n0: the reference requires n0 >= k (graphgp/tree.py:56-57); requests are built with
n0 = max(k, min(256, N // 100)).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

OPS = ("generate", "inverse", "logdet")


@dataclass
class Request:
    rid: int
    op: str                      # "generate" | "inverse" | "logdet"
    points: np.ndarray           # (n, d) float32
    k: int
    n0: int
    bins: np.ndarray             # kernel table
    vals: np.ndarray
    payload: Optional[np.ndarray] = None  # xi (generate) or values (inverse), (n,) float32
    arrival: float = 0.0
    graph_key: Optional[object] = None   # requests naming the same key share one resident graph
    table_key: Optional[object] = None   # ... and one resident kernel table

    @property
    def n(self) -> int:
        return int(self.points.shape[0])


@dataclass
class Result:
    rid: int
    op: str
    n: int
    output: object
    arrival: float
    start: float
    end: float
    status: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.end - self.arrival


def footprint_bytes(n: int, d: int, k: int, n0: int, n_bins: int, dtype_bytes: int = 4) -> int:
    """Device bytes a request holds while in flight: inputs and graph (points, indices, neighbours, depths,
    offsets), outputs, and the larger of the graph-build and operation workspaces (workspace sizes from
    ggp_workspace_size)."""
    from . import _lib

    lib = _lib.load()
    ops = _lib.OPS
    b = int(dtype_bytes)
    graph_ws = lib.ggp_workspace_size(ops["BUILD_GRAPH"], n, d, n0, k, 2, 1, b)
    op_ws = max(lib.ggp_workspace_size(ops[o], n, d, n0, k, n_bins, n + 1, b)
                for o in ("GENERATE", "GENERATE_INV", "GENERATE_LOGDET"))
    resident = 2 * b * n * d + 4 * n * (k + 4) + 2 * b * n + 4 * (n + 1)
    return int(resident + max(graph_ws, op_ws) + (1 << 20))


class Scheduler:
    """Admission and slot logic, independent of the device: ``slots`` worker threads take requests in arrival
    order; the head of the queue is admitted when its footprint fits in ``budget`` minus the footprints in
    flight, or when nothing is in flight (a request larger than the whole budget then runs alone).
    ``process(req, slot_state)`` does the work; ``slot_init()`` builds each worker's state (its stream)."""

    def __init__(self, slots: int, budget: int, footprint, process, slot_init=lambda: None):
        if slots < 1:
            raise ValueError("slots must be >= 1")
        self.slots, self.budget = int(slots), int(budget)
        self.footprint, self.process, self.slot_init = footprint, process, slot_init
        self.peak_in_use = 0
        self.peak_in_flight = 0
        self.admission_order = []

    def run(self, requests, realtime: bool = True):
        """Serve ``requests``. With ``realtime`` a request becomes visible only at its arrival time (seconds
        after the start); otherwise all are queued at once. Returns (results sorted by rid, wall seconds)."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        foot = {r.rid: int(self.footprint(r)) for r in reqs}
        pending = deque()
        results = []
        cv = threading.Condition()
        state = {"in_use": 0, "in_flight": 0, "closed": False, "error": None}
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        def arrivals():
            for r in reqs:
                if realtime:
                    dt = r.arrival - now()
                    if dt > 0:
                        time.sleep(dt)
                with cv:
                    if state["error"] is not None:
                        break
                    pending.append(r)
                    cv.notify_all()
            with cv:
                state["closed"] = True
                cv.notify_all()

        def admit():
            """Blocks until the head request can be admitted; None when the stream is over or failed."""
            with cv:
                while True:
                    if state["error"] is not None:
                        return None
                    if pending:
                        need = foot[pending[0].rid]
                        if state["in_flight"] == 0 or state["in_use"] + need <= self.budget:
                            r = pending.popleft()
                            state["in_use"] += need
                            state["in_flight"] += 1
                            self.peak_in_use = max(self.peak_in_use, state["in_use"])
                            self.peak_in_flight = max(self.peak_in_flight, state["in_flight"])
                            self.admission_order.append(r.rid)
                            return r
                    elif state["closed"]:
                        return None
                    cv.wait(0.05)

        def worker():
            try:
                slot = self.slot_init()
            except Exception as exc:  # noqa: BLE001 -- reported by run()
                with cv:
                    state["error"] = exc
                    cv.notify_all()
                return
            while True:
                r = admit()
                if r is None:
                    return
                start = now()
                try:
                    out, st = self.process(r, slot)
                except Exception as exc:  # noqa: BLE001 -- reported by run()
                    with cv:
                        state["error"] = exc
                        cv.notify_all()
                    return
                end = now()
                with cv:
                    results.append(Result(r.rid, r.op, r.n, out, r.arrival, start, end, st))
                    state["in_use"] -= foot[r.rid]
                    state["in_flight"] -= 1
                    cv.notify_all()

        threads = [threading.Thread(target=worker, daemon=True) for _ in range(self.slots)]
        feeder = threading.Thread(target=arrivals, daemon=True)
        for t in threads:
            t.start()
        feeder.start()
        feeder.join()
        for t in threads:
            t.join()
        if state["error"] is not None:
            raise state["error"]
        results.sort(key=lambda x: x.rid)
        return results, now()


class _Slot:
    """A worker's device state: its CUDA stream and pinned host staging buffers. Uploads go numpy -> pinned
    buffer (a host memcpy) -> device on the slot's stream, and results come back into a pinned buffer; copies
    from or to pageable memory would all pass through the driver's one staging path and serialise the slots. A
    slot runs one request at a time and waits for its result before the next one reuses the buffers."""

    def __init__(self, torch, device, stream=None):
        self.torch = torch
        self.stream = stream if stream is not None else torch.cuda.Stream(device=device)
        self._bufs = {}
        self.native = {}  # device and pinned blocks of the one-call host path (graphgp_cuda.request_host)

    def pinned(self, name, numel, dtype):
        t = self._bufs.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = self.torch.empty(max(int(numel), 1024), dtype=dtype, pin_memory=True)
            self._bufs[name] = t
        return t[:numel]

    def upload(self, name, array, dtype, device):
        """A numpy array -> a device tensor of the same shape, through this slot's pinned buffer."""
        a = np.ascontiguousarray(array)
        host = self.pinned(name, a.size, dtype).view(a.shape)
        host.copy_(self.torch.from_numpy(a))
        return host.to(device, non_blocking=True)

    def download(self, name, tensor):
        """A device tensor -> numpy (a copy), through this slot's pinned buffer; waits on the slot's stream."""
        host = self.pinned(f"{name}_{tensor.dtype}", tensor.numel(), tensor.dtype).view(tensor.shape)
        host.copy_(tensor, non_blocking=True)
        self.stream.synchronize()
        return host.numpy().copy()


class Engine:
    """The device side: each slot owns a CUDA stream; a request uploads its inputs, builds its graph, runs its
    operation and reads its result back on that stream. Graphs (``Request.graph_key``) and kernel tables
    (``Request.table_key``) named by a key stay resident on the device for later requests."""

    def __init__(self, device=None, slots: int = 16, hbm_budget: int = 32 << 30, tau: Optional[float] = None,
                 dtype=None, fused: bool = True):
        import torch

        from . import graphgp_cuda as gc

        self.torch = torch
        self.gc = gc
        self.device = torch.device(device or "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.slots = int(slots)
        self.budget = int(hbm_budget)
        self.tau = tau  # None: each operation's default threshold
        self.fused = fused  # requests with nothing resident: one native call (ggp_request_*) or separate calls
        self.dtype = dtype or torch.float32
        if self.dtype not in (torch.float32, torch.float64):
            raise TypeError("dtype must be torch.float32 or torch.float64")
        self._np = np.float32 if self.dtype == torch.float32 else np.float64
        self._graphs = {}
        self._tables = {}
        self._lock = threading.Lock()
        self.last_scheduler = None

    def _slot_init(self):
        torch = self.torch
        torch.cuda.set_device(self.device)
        return _Slot(torch, self.device)

    def _cached(self, cache, key, make):
        if key is None:
            return make()
        with self._lock:
            v = cache.get(key)
        if v is None:
            v = make()
            with self._lock:
                v = cache.setdefault(key, v)
        return v

    def process(self, req: Request, slot=None):
        """One request on ``slot`` (a worker's slot, a CUDA stream, or None for the current stream); returns
        (output, status dict)."""
        torch, gc, dev = self.torch, self.gc, self.device
        if not isinstance(slot, _Slot):
            slot = _Slot(torch, dev, stream=slot or torch.cuda.current_stream(dev))
        dt = self.dtype
        with torch.cuda.stream(slot.stream), torch.cuda.nvtx.range(f"request {req.rid} {req.op} n={req.n}"):

            def make_graph():
                P = slot.upload("points", req.points, dt, dev)
                return gc.build_graph(P, n0=req.n0, k=req.k, return_offsets=True)

            def make_table():
                return slot.upload("bins", req.bins, dt, dev), slot.upload("vals", req.vals, dt, dev)

            if req.op not in OPS:
                raise ValueError(f"unknown op {req.op!r}")
            if self.fused and req.graph_key is None and req.table_key is None:
                # nothing resident to reuse: staging, upload, graph build, operation, readback and status in one
                # native call that holds no Python lock
                return gc.request_host(req.op, np.asarray(req.points, self._np), req.n0, req.k, req.bins, req.vals,
                                       req.payload if req.op != "logdet" else None, tau=self.tau, buffers=slot.native,
                                       device=dev)
            # a resident graph and / or table: separate calls on the device tensors
            x = slot.upload("payload", req.payload, dt, dev) if req.op != "logdet" else None
            gp, gi, gn, _, offs = self._cached(self._graphs, req.graph_key, make_graph)
            B, V = self._cached(self._tables, req.table_key, make_table)
            if req.op == "generate":
                r = gc.generate(gp, gi, gn, offs, B, V, x, tau=self.tau)
            elif req.op == "inverse":
                r = gc.generate_inv(gp, gi, gn, offs, B, V, x, tau=self.tau)
            else:
                r = gc.generate_logdet(gp, gn, offs, B, V, tau=self.tau)
            out = slot.download("out", r.reshape(-1))
            out = float(out[0]) if req.op == "logdet" else out
            return out, gc.last_status()

    def footprint(self, req: Request) -> int:
        return footprint_bytes(req.n, req.points.shape[1], req.k, req.n0, len(req.bins), self.dtype.itemsize)

    def run(self, requests, realtime: bool = True):
        """Serve ``requests``; returns (results sorted by rid, summary dict)."""
        sch = Scheduler(self.slots, self.budget, self.footprint, lambda r, s: self.process(r, s), self._slot_init)
        self.last_scheduler = sch
        results, wall = sch.run(requests, realtime)
        summary = summarize(results, wall)
        summary.update(slots=self.slots, hbm_budget=self.budget, peak_in_use=sch.peak_in_use,
                       peak_in_flight=sch.peak_in_flight)
        return results, summary


def summarize(results, wall):
    lat = np.array([r.latency for r in results]) * 1e3
    pts = sum(r.n for r in results)
    by_op = {op: int(sum(r.op == op for r in results)) for op in OPS}
    return {
        "requests": len(results),
        "wall_s": wall,
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_ms": float(lat.mean()) if len(lat) else None,
        "requests_per_s": len(results) / wall if wall > 0 else None,
        "points_per_s": pts / wall if wall > 0 else None,
        "op_mix": by_op,
    }


def synthetic_stream(n_requests=4096, rate=2000.0, seed=0, median_n=30000, sigma=1.0, n_min=1000, n_max=1000000,
                     n_bins=1000):
    """The serving workload: Poisson arrivals at ``rate`` req/s; N lognormal (median 30,000, log-sd 1) clipped to
    [1e3, 1e6]; d uniform in {2, 3}; k uniform in {8, 16, 32}; n0 = max(k, min(256, N // 100)); standard
    normal float32 points; an RBF table per request (scale U(0.05, 0.5), r = 0 plus ``n_bins`` - 1 log bins on
    [1e-4, 10]); op mix 70 % generate, 20 % inverse, 10 % logdet."""
    from . import extras

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    reqs = []
    for i in range(n_requests):
        n = int(np.clip(rng.lognormal(np.log(median_n), sigma), n_min, n_max))
        d = int(rng.integers(2, 4))
        k = int(rng.choice([8, 16, 32]))
        n0 = max(k, min(256, n // 100))
        op = rng.choice(OPS, p=[0.7, 0.2, 0.1])
        pts = rng.standard_normal((n, d)).astype(np.float32)
        bins, vals = extras.rbf_kernel(variance=1.0, scale=float(rng.uniform(0.05, 0.5)), r_min=1e-4, r_max=10.0,
                                       n_bins=n_bins, jitter=1e-4)
        payload = rng.standard_normal(n).astype(np.float32) if op != "logdet" else None
        reqs.append(Request(i, str(op), pts, k, n0, bins, vals, payload, float(t[i])))
    return reqs
