"""Serving loop on the GPU: every request served in the mix (overlapping on several streams, admitted by
footprint) gives the same result as the same request served alone, and small requests match the FP64 oracle.

Tolerance for alone-vs-mix: values of generate / inverse bit-identical (each point's arithmetic does not depend
on scheduling); log-determinant within 1e-12 relative (an FP64 sum of per-block partials)."""
import numpy as np
import pytest

from graphgp_b200 import serving as sv

pytestmark = pytest.mark.gpu


def _stream(n_requests, seed, median_n=3000, n_max=40000):
    return sv.synthetic_stream(n_requests=n_requests, rate=4000.0, seed=seed, median_n=median_n, n_min=1000,
                               n_max=n_max, n_bins=1000)


def _same(a, b, op):
    if op == "logdet":
        return abs(a - b) <= 1e-12 * max(1.0, abs(b)) or (np.isnan(a) and np.isnan(b))
    return np.array_equal(a, b, equal_nan=True)


def test_mix_equals_alone(cuda_device):
    reqs = _stream(64, seed=11)
    eng = sv.Engine(cuda_device, slots=8, hbm_budget=8 << 30)
    mixed, summary = eng.run(reqs, realtime=True)
    assert summary["requests"] == 64 and summary["peak_in_flight"] >= 2
    alone = sv.Engine(cuda_device, slots=1)
    for r, m in zip(reqs, mixed):
        out, st = alone.process(r)
        assert st["error"] == 0 and m.status["error"] == 0
        assert _same(m.output, out, r.op), (r.rid, r.op, r.n, r.k)


def test_budget_limits_concurrency(cuda_device):
    reqs = _stream(24, seed=12, median_n=20000, n_max=100000)
    foot = [sv.footprint_bytes(r.n, r.points.shape[1], r.k, r.n0, len(r.bins)) for r in reqs]
    budget = int(2.5 * max(foot))
    eng = sv.Engine(cuda_device, slots=16, hbm_budget=budget)
    res, summary = eng.run(reqs, realtime=False)
    assert summary["peak_in_use"] <= budget
    assert eng.last_scheduler.admission_order == sorted(eng.last_scheduler.admission_order)
    assert all(r.status["error"] == 0 for r in res)


def test_resident_graph_and_table_reuse(cuda_device):
    base = _stream(1, seed=13)[0]
    rng = np.random.default_rng(0)
    reqs = []
    for i in range(6):
        op = ("generate", "inverse", "logdet")[i % 3]
        pay = rng.standard_normal(base.n).astype(np.float32) if op != "logdet" else None
        reqs.append(sv.Request(i, op, base.points, base.k, base.n0, base.bins, base.vals, pay, 0.0, graph_key="g",
                               table_key="t"))
    eng = sv.Engine(cuda_device, slots=3)
    res, _ = eng.run(reqs, realtime=False)
    assert len(eng._graphs) == 1 and len(eng._tables) == 1
    fresh = sv.Engine(cuda_device, slots=1)
    for r, m in zip(reqs, res):
        r2 = sv.Request(r.rid, r.op, r.points, r.k, r.n0, r.bins, r.vals, r.payload)
        out, _ = fresh.process(r2)
        assert _same(m.output, out, r.op)


def _oracle_requests(dtype=np.float32):
    from oracle import graph as og
    from oracle import refine as orf

    pool = [r for r in _stream(200, seed=14, median_n=1500, n_max=3000) if r.k <= 16]
    reqs = [r for op in sv.OPS for r in [q for q in pool if q.op == op][:2]]
    assert len(reqs) == 6
    graphs = {r.rid: og.build_graph(r.points.astype(dtype), n0=r.n0, k=r.k) for r in reqs}
    for r in reqs:
        if r.op == "inverse":  # invert a sample of the process
            r.payload = orf.generate(graphs[r.rid], (r.bins, r.vals), r.payload.astype(np.float64)).astype(np.float32)
    return reqs, graphs


def _check_vs_oracle(reqs, graphs, res, tol, tol_inv, dtype):
    from oracle import refine as orf

    from conftest import rel_err
    from helpers import as_inputs

    by_rid = {m.rid: m for m in res}
    for r in reqs:
        # the FP64 oracle on the table as the engine hands it to the kernels (rounded to their dtype)
        m, g, cov = by_rid[r.rid], graphs[r.rid], as_inputs((r.bins, r.vals), dtype)
        if r.op == "generate":
            assert rel_err(m.output, orf.generate(g, cov, r.payload.astype(np.float64))) < tol, r.rid
        elif r.op == "inverse":
            assert rel_err(m.output, orf.generate_inv(g, cov, r.payload.astype(np.float64))) < tol_inv, r.rid
        else:
            ref = orf.generate_logdet(g, cov)
            assert abs(m.output - ref) <= tol * abs(ref), r.rid


def test_requests_match_oracle_f32(cuda_device):
    """Served FP32 requests against the FP64 oracle: generate, inverse and log-determinant within 1e-4 relative.

    These RBF tables (length scale up to 0.5 on standard-normal points) put most pivot ratios near the jitter
    (1e-4); an FP32 inverse divides the FP32 rounding of the conditional mean by the conditional standard
    deviation (NumPy float32 is 3e-4 off on one of these requests), so the inverse re-conditions every point
    whose pivot ratio is below 3e-3 in FP64 (the engine's default thresholds). The oracle runs on the table
    rounded to FP32, the inputs the FP32 kernels receive."""
    reqs, graphs = _oracle_requests()
    res, _ = sv.Engine(cuda_device, slots=4).run(reqs, realtime=False)
    _check_vs_oracle(reqs, graphs, res, 1e-4, 1e-4, np.float32)


def test_requests_match_oracle_f64(cuda_device):
    """The same requests served in FP64: every operation within 1e-8 relative of the oracle."""
    import torch

    reqs, graphs = _oracle_requests(np.float64)
    res, _ = sv.Engine(cuda_device, slots=4, dtype=torch.float64).run(reqs, realtime=False)
    _check_vs_oracle(reqs, graphs, res, 1e-8, 1e-8, np.float64)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_native_request_equals_separate_calls(cuda_device, dtype):
    """ggp_request_* (graph build + operation in one call) gives exactly what build_graph followed by
    generate / generate_inv / generate_logdet gives."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    dt = getattr(torch, dtype)
    r = _stream(1, seed=21, median_n=5000)[0]
    P = torch.as_tensor(r.points, device=cuda_device).to(dt)
    B = torch.as_tensor(r.bins, device=cuda_device).to(dt)
    V = torch.as_tensor(r.vals, device=cuda_device).to(dt)
    x = torch.as_tensor(np.random.default_rng(0).standard_normal(r.n), device=cuda_device).to(dt)
    gp, gi, gn, _, offs = gc.build_graph(P, n0=r.n0, k=r.k, return_offsets=True)
    ref = {"generate": gc.generate(gp, gi, gn, offs, B, V, x), "inverse": gc.generate_inv(gp, gi, gn, offs, B, V, x),
           "logdet": gc.generate_logdet(gp, gn, offs, B, V)}
    for op in ("generate", "inverse", "logdet"):
        out = gc.request(op, P, r.n0, r.k, B, V, None if op == "logdet" else x)
        assert gc.last_status()["error"] == 0
        if op == "logdet":
            assert abs(float(out) - float(ref[op])) <= 1e-12 * abs(float(ref[op]))
        else:
            assert torch.equal(out, ref[op]), op


def test_concurrent_requests_with_different_table_sizes(cuda_device):
    """Requests whose kernel tables differ in size (so their launches need different shared memory) run on 8
    streams at once, and each still gives the result it gives alone."""
    base = _stream(24, seed=31, median_n=4000, n_max=20000)
    reqs = []
    for i, r in enumerate(base):
        nb = (1000, 4097, 257)[i % 3]
        from graphgp_b200 import extras

        bins, vals = extras.rbf_kernel(variance=1.0, scale=0.2, r_min=1e-4, r_max=10.0, n_bins=nb, jitter=1e-4)
        reqs.append(sv.Request(r.rid, r.op, r.points, r.k, r.n0, bins, vals, r.payload, 0.0))
    res, _ = sv.Engine(cuda_device, slots=8).run(reqs, realtime=False)
    alone = sv.Engine(cuda_device, slots=1)
    for r, m in zip(reqs, res):
        out, st = alone.process(r)
        assert m.status["error"] == 0 and st["error"] == 0
        assert _same(m.output, out, r.op), (r.rid, len(r.bins))


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_request_host_equals_device_request(cuda_device, dtype):
    """The one-call host path (ggp_request_host_*: pinned staging, upload, build, operation, readback, status)
    gives what the device-tensor request gives on the same inputs (bit-identical values; the log-determinant's
    FP64 partial sums within 1e-12)."""
    import torch

    from graphgp_b200 import graphgp_cuda as gc

    tdt = getattr(torch, dtype)
    buffers = {}
    for r in _stream(6, seed=5):
        pts = np.asarray(r.points, dtype)
        P = torch.as_tensor(pts, device=cuda_device)
        B = torch.as_tensor(np.asarray(r.bins), dtype=tdt, device=cuda_device)
        V = torch.as_tensor(np.asarray(r.vals), dtype=tdt, device=cuda_device)
        pay = None if r.op == "logdet" else np.asarray(r.payload, dtype)
        dev_out = gc.request(r.op, P, r.n0, r.k, B, V, None if pay is None else torch.as_tensor(pay, device=cuda_device))
        ref = float(dev_out.item()) if r.op == "logdet" else dev_out.cpu().numpy()
        out, st = gc.request_host(r.op, pts, r.n0, r.k, r.bins, r.vals, pay, buffers=buffers, device=cuda_device)
        assert st["error"] == 0
        if r.op != "logdet":
            assert out.dtype == np.dtype(dtype)
        assert _same(out, ref, r.op)
