#!/usr/bin/env python
"""Benchmark of the GraphGP hot path on B200: FP32 ``generate`` (FP64 dense root) at the precision-at-scale
workload -- N = 16,777,216 points in d = 3 (unit direction x 10^U(-3, 0), float32, seed 99), n0 = 1024,
k = 16, Matern-3/2 (variance 1, cutoff 0.05) tabulated at r = 0 plus 2048 log bins on [1e-6, 4],
jitter 1e-5, xi ~ N(0, 1). The graph is built once on the GPU (untimed, reported separately); a step is
one ``generate`` of all N points with the inputs resident in HBM (inputs larger than L2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n N]

Prints one JSON line (rank 0). With --gpus N > 1 (torchrun) every rank runs an independent replica on its
own GPU ("replicas only": generate has no shardable exchange step); value = all ranks' points / max time.
``--impl reference`` times the CPU restatement of the reference's algorithm (the NumPy oracle) on the host
cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec generate+grad, FP32 vs FP64 at ≤1e-4 rel err; p50/p99 request latency"
WORKLOAD = dict(name="generate, precision at scale", n=1 << 24, d=3, n0=1024, k=16, kernel="matern-3/2",
                cutoff=0.05, r_min=1e-6, r_max=4.0, n_bins=2049, jitter=1e-5, seed=99)
BYTES_PER_POINT = 4 * WORKLOAD["k"] * (WORKLOAD["d"] + 2) + 4 * WORKLOAD["d"] + 8  # 340 B (k=16, d=3)


def flops_per_point(k, d):
    """Algorithmic flops of one refined point: pair distances + interpolation, Cholesky, triangular solve, mean and
    value: (k+1)(k+2)/2 (3d+4) + 2(k+1)^3/3 + k(k+1) + 2k + 2 (5,570 at k = 16, d = 3)."""
    return (k + 1) * (k + 2) / 2 * (3 * d + 4) + 2 * (k + 1) ** 3 / 3 + k * (k + 1) + 2 * k + 2


FLOPS_PER_POINT = flops_per_point(WORKLOAD["k"], WORKLOAD["d"])


def fma_peaks(dev):
    """Measured CUDA-core peaks (TFLOP/s) from ggp_fma_probe: FP32 (the better of fma.rn.f32 and the packed
    fma.rn.f32x2) and FP64, each the best of 3 timed launches of 148 x 8 blocks after one warm-up, CUDA events on
    the launching stream, default clocks."""
    import ctypes as C

    import torch

    from graphgp_b200 import _lib

    lib = _lib.load()
    sink = torch.empty(4096, dtype=torch.uint8, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    for kind, name, iters in ((0, "fp32", 4096), (1, "fp32x2", 4096), (2, "fp64", 2048)):
        fl = C.c_double(0)
        best = 0.0
        for rep in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(lib.ggp_fma_probe(kind, 148 * 8, iters, C.byref(fl), C.c_void_p(sink.data_ptr()), sink.numel(),
                                         s), "ggp_fma_probe")
            e1.record()
            torch.cuda.synchronize()
            if rep:
                best = max(best, fl.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        out[name] = best
    out["fp32_best"] = max(out["fp32"], out["fp32x2"])
    return out


def synth_points(n, d=3, seed=99):
    """Unit direction times radius 10^U(-3, 0) (heavy dynamic range), float32."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, d))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * 10.0 ** rng.uniform(-3, 0, (n, 1))).astype(np.float32)


def table():
    from graphgp_b200 import extras

    w = WORKLOAD
    return extras.matern_kernel(p=1, variance=1.0, cutoff=w["cutoff"], r_min=w["r_min"], r_max=w["r_max"],
                                n_bins=w["n_bins"], jitter=w["jitter"])


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons in the background during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl" if _cuda_ok() else "gloo", timeout=timedelta(seconds=300))
    return world, rank, local


def _cuda_ok():
    import torch

    return torch.cuda.is_available()


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------------------------------------
# FP64 comparators
# ------------------------------------------------------------------------------------------------
def fp64_fastjit_generate(P, I, NB, offsets, bins, vals, xi, chunk=1 << 19):
    """The plain FP64-GPU form shaped like the reference's fast_jit path (refine.py:123-145): materialise
    the (k+1)^2 covariance of every point in float64, batched Cholesky (torch / cuSOLVER), mean_vec =
    solve(L11^T, l21), then the batch scan of gathers. Dense root in FP64 as well. Comparator only."""
    import torch

    n = P.shape[0]
    n0 = n - NB.shape[0]
    k = NB.shape[1]
    P64 = P.double()
    b64 = bins.double()
    v64 = vals.double()

    def interp(r):
        i = torch.clamp(torch.searchsorted(b64, r, right=True), 1, len(b64) - 1)
        x0, x1 = b64[i - 1], b64[i]
        f0, f1 = v64[i - 1], v64[i]
        f = f0 + (r - x0) / (x1 - x0) * (f1 - f0)
        f = torch.where(r < b64[0], v64[0], f)
        return torch.where(r > b64[-1], v64[-1], f)

    mean_vec = torch.empty((n - n0, k), dtype=torch.float64, device=P.device)
    std = torch.empty(n - n0, dtype=torch.float64, device=P.device)
    for s in range(0, n - n0, chunk):
        e = min(n - n0, s + chunk)
        joint = torch.cat([P64[NB[s:e].long()], P64[n0 + s:n0 + e, None]], dim=1)
        K = interp(torch.cdist(joint, joint))
        L = torch.linalg.cholesky(K)
        mean_vec[s:e] = torch.linalg.solve_triangular(L[:, :k, :k].transpose(1, 2), L[:, k, :k, None],
                                                      upper=True)[..., 0]
        std[s:e] = L[:, k, k]
        del joint, K, L
    xi64 = xi.double()[I.long()]
    K0 = interp(torch.cdist(P64[:n0], P64[:n0]))
    values = torch.zeros(n, dtype=torch.float64, device=P.device)
    values[:n0] = torch.linalg.cholesky(K0) @ xi64[:n0]
    NBl = NB.long()
    for b in range(1, len(offsets)):
        s, e = offsets[b - 1], offsets[b]
        rows = slice(s - n0, e - n0)
        values[s:e] = (mean_vec[rows] * values[NBl[rows]]).sum(1) + std[rows] * xi64[s:e]
    out = torch.empty_like(values)
    out[I.long()] = values
    return out


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch

    from graphgp_b200 import _lib
    from graphgp_b200 import graphgp_cuda as gc

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOAD
    n = args.n or w["n"]
    lib = _lib.load()
    pts = synth_points(n, w["d"], w["seed"])
    bins, vals = table()
    P = torch.as_tensor(pts, device=dev)
    B = torch.as_tensor(bins, dtype=torch.float32, device=dev)
    V = torch.as_tensor(vals, dtype=torch.float32, device=dev)
    xi_host = np.random.default_rng(w["seed"] + 1).standard_normal(n).astype(np.float32)
    XI = torch.as_tensor(xi_host, device=dev)

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    # graph (one-time, untimed for the metric)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    gp, gi, gn, gd, offs = gc.build_graph(P, n0=w["n0"], k=w["k"], return_offsets=True)
    e1.record()
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1)
    OF = torch.as_tensor(offs, dtype=torch.int32, device=dev)

    step = lambda: gc.generate(gp, gi, gn, OF, B, V, XI)  # noqa: E731
    for _ in range(args.warmup):
        out = step()
    torch.cuda.synchronize()
    st = gc.last_status()
    launches0 = lib.ggp_launch_count()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(args.steps):
            out = step()
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
    launches = (lib.ggp_launch_count() - launches0) / args.steps
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    # dominant kernel: the refinement kernel in generate mode (graphgp_cuda.refine = prologue + that kernel)
    init = out[gi[: w["n0"]].long()].contiguous()
    xr = XI[gi[w["n0"]:].long()].contiguous()
    for _ in range(2):
        gc.refine(gp, gn, OF, B, V, init, xr)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(args.steps):
        gc.refine(gp, gn, OF, B, V, init, xr)
    e1.record()
    torch.cuda.synchronize()
    kern_ms = e0.elapsed_time(e1) / args.steps

    # end to end through the public API with host buffers: pinned xi in, values out
    xi_pin = torch.from_numpy(xi_host).pin_memory()
    out_pin = torch.empty(n, dtype=torch.float32).pin_memory()
    for _ in range(2):
        out_pin.copy_(gc.generate(gp, gi, gn, OF, B, V, xi_pin.to(dev, non_blocking=True)), non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(args.steps):
        x_d = xi_pin.to(dev, non_blocking=True)
        out_pin.copy_(gc.generate(gp, gi, gn, OF, B, V, x_d), non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    # generate + gradient through autograd: loss = 0.5|generate(xi) - y|^2 + logdet, loss.backward() (one adjoint
    # sweep for both terms, w.r.t. xi and the table values)
    import graphgp_b200 as gg

    Y = out + 0.01 * torch.randn(n, generator=torch.Generator(device=dev).manual_seed(5), device=dev)
    graph = gg.Graph(gp, gn, OF, gi)
    XG = XI.clone().requires_grad_(True)
    VG = V.clone().requires_grad_(True)

    def grad_step():
        XG.grad = None
        VG.grad = None
        v, ld = gg.generate_and_logdet(graph, (B, VG), XG)
        loss = 0.5 * torch.sum((v - Y) ** 2) + ld
        loss.backward()
        return XG.grad, VG.grad

    for _ in range(2):
        grad_step()
    torch.cuda.synchronize()
    gst = gc.last_status()
    barrier(world)
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(args.steps):
        grad_step()
    e1.record()
    torch.cuda.synchronize()
    grad_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)

    extra = {"generate_grad": {"value": n * world / (grad_ms * 1e-3), "unit": "points/s", "ms_per_step": grad_ms,
                               "step": "loss = 0.5|generate(xi) - y|^2 + generate_logdet, loss.backward() through "
                                       "graphgp_b200.generate_and_logdet (forward values and logdet, one adjoint "
                                       "sweep w.r.t. xi and the table values)",
                               "status_error": gst["error"] if gst else None}}
    # inverse and log-determinant of the same workload (no dependency waits)
    for name, fn in (("inverse", lambda: gc.generate_inv(gp, gi, gn, OF, B, V, out)),
                     ("logdet", lambda: gc.generate_logdet(gp, gn, OF, B, V))):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        t_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
        sst = gc.last_status()
        extra[name] = {"value": n * world / (t_ms * 1e-3), "unit": "points/s", "ms_per_step": t_ms,
                       "fp64_points": sst["fallback_count"] if sst else None}
    if rank == 0 and not args.quick:
        extra.update(comparisons(args, dev, gp, gi, gn, offs, OF, B, V, XI, pts, bins, vals, out, ms))
    if rank == 0 and args.serving_requests > 0:
        extra["serving"] = serving(dev, args.serving_requests)
    if rank == 0 and args.fd_directions > 0:
        extra["differentiation"] = differentiation(dev, n_dirs=args.fd_directions)

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = BYTES_PER_POINT * (n - w["n0"]) / (kern_ms * 1e-3) / 1e9
    traffic = read_traffic(n - w["n0"])
    fma = fma_peaks(dev)
    achieved_tf = FLOPS_PER_POINT * (n - w["n0"]) / (kern_ms * 1e-3) / 1e12
    fp32_frac = achieved_tf / fma["fp32_best"]
    hbm_frac = achieved / hbm
    line = {
        "metric": METRIC,
        "value": n * world / (ms * 1e-3),
        "unit": "points/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (FP64 dense root, FP64 logdet sums, FP64 re-conditioning below pivot ratio 1e-5)",
        "data": "synthetic (seeded NumPy: unit direction x 10^U(-3,0), float32; xi N(0,1))",
        "config": {"workload": w["name"], "n_points": n, "d": w["d"], "n0": w["n0"], "k": w["k"],
                   "kernel": f"{w['kernel']} cutoff {w['cutoff']}, r=0 + {w['n_bins'] - 1} log bins on "
                             f"[{w['r_min']}, {w['r_max']}], jitter {w['jitter']}",
                   "batches": len(offs) - 1, "graph_build_ms": graph_ms, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (points 201 MB, neighbours 1.07 GB)"},
        "e2e": {"value": n * world / (e2e_ms * 1e-3), "unit": "points/s",
                "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * n, "ms_per_step": e2e_ms},
        "roofline": {"bound": "fp32" if fp32_frac >= hbm_frac else "hbm",
                     "achieved": achieved_tf if fp32_frac >= hbm_frac else achieved,
                     "peak": fma["fp32_best"] if fp32_frac >= hbm_frac else hbm,
                     "unit": "TFLOP/s" if fp32_frac >= hbm_frac else "GB/s",
                     "frac": max(fp32_frac, hbm_frac),
                     "fp32_frac": fp32_frac, "achieved_fp32_tflops": achieved_tf,
                     "peak_fp32_tflops": fma["fp32_best"], "peak_fp32_ffma_tflops": fma["fp32"],
                     "peak_fp32_ffma2_tflops": fma["fp32x2"], "peak_fp64_tflops": fma["fp64"],
                     "hbm_frac": hbm_frac, "achieved_hbm_gbs": achieved, "peak_hbm_gbs": hbm,
                     "traffic": traffic, "kernel": REFINE_KERNEL,
                     "traffic_source": TRAFFIC_SOURCE,
                     "kernel_ms": kern_ms, "algorithmic_bytes_per_point": BYTES_PER_POINT,
                     "algorithmic_flops_per_point": FLOPS_PER_POINT,
                     "peak_source": "fp32/fp64: ggp_fma_probe measured in this run (of measured); hbm: "
                                    + ("MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback")},
        "gpu_launches": launches,
        "fallback_points": st["fallback_count"] if st else None,
    }
    line.update(extra)
    if rank == 0:
        line["clocks"] = clk.summary()
        if not args.quick and "_subset" in line:
            line["cpu_baseline"] = cpu_baseline(line.pop("_subset"), bins, vals)
        if args.largest:
            del gp, gi, gn, OF, XI, P, out, Y, graph, XG, VG
            torch.cuda.empty_cache()
            line["largest"] = largest(dev, n=args.largest_n, steps=1)
        print(json.dumps(line), flush=True)


def largest_points(n, seed=2027, block=1 << 20):
    """Points of the largest-instance workload: a mixture of 64 Gaussian clusters (centres uniform in [-1, 1]^3,
    per-cluster sigma 10^U(-3, -1), 90 % of the points) plus 10 % uniform background in [-1, 1]^3, float32.
    Generated in blocks of 2^20 points, block b from seed + 1 + b, so the first 2^20 points (the parity
    subset) are the same whatever n is."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, (64, 3))
    sigmas = 10.0 ** rng.uniform(-3.0, -1.0, 64)
    out = np.empty((n, 3), np.float32)
    for b0 in range(0, n, block):
        m = min(block, n - b0)
        r = np.random.default_rng(seed + 1 + b0 // block)
        c = r.integers(0, 64, m)
        x = centres[c] + sigmas[c, None] * r.standard_normal((m, 3))
        bg = r.random(m) < 0.1
        x[bg] = r.uniform(-1.0, 1.0, (int(bg.sum()), 3))
        out[b0:b0 + m] = x
    return out


def differentiation(dev, n_dirs=64, steps=5, warmup=3, n=4194304):
    """Generate + gradient on the differentiation workload: N = 4,194,304 points uniform in [0, 1]^2 (float32),
    n0 = 256, k = 20, RBF scale 0.1 with r = 0 + 1,000 log bins on [1e-5, 1.5] (1,001 values), jitter 1e-4;
    y = generate(xi*) + 0.01 N(0, 1); loss 0.5 |generate(xi) - y|^2 + logdet. Times the FP32 step (forward,
    residual, adjoint w.r.t. xi and the table values) and checks <grad, u> against central differences of the
    FP64 forward along n_dirs random directions: half move xi only (u standard normal, unit norm; the loss is
    quadratic in xi, so differences with step 1e-3 are exact up to rounding), half move the table only
    (u = 1e-3 vals * N(0, 1), a relative perturbation that keeps every joint covariance positive definite under
    the jitter); there the loss is far from quadratic, so the differences are taken with steps 1e-3 and 1e-5."""
    import torch

    from graphgp_b200 import extras
    from graphgp_b200 import graphgp_cuda as gc

    rng = np.random.default_rng(2024)
    pts = rng.uniform(0.0, 1.0, (n, 2)).astype(np.float32)
    bins, vals = extras.rbf_kernel(variance=1.0, scale=0.1, r_min=1e-5, r_max=1.5, n_bins=1001, jitter=1e-4)
    P = torch.as_tensor(pts, device=dev)
    gp, gi, gn, _, offs = gc.build_graph(P, n0=256, k=20, return_offsets=True)
    OF = torch.as_tensor(offs, dtype=torch.int32, device=dev)
    B = torch.as_tensor(bins, dtype=torch.float32, device=dev)
    V = torch.as_tensor(vals, dtype=torch.float32, device=dev)
    xs = torch.as_tensor(rng.standard_normal(n).astype(np.float32), device=dev)
    y = gc.generate(gp, gi, gn, OF, B, V, xs) + 0.01 * torch.as_tensor(rng.standard_normal(n).astype(np.float32),
                                                                        device=dev)
    xi = torch.as_tensor(rng.standard_normal(n).astype(np.float32), device=dev)
    import graphgp_b200 as gg

    graph = gg.Graph(gp, gn, OF, gi)
    XG = xi.clone().requires_grad_(True)
    VG = V.clone().requires_grad_(True)

    def step():
        # loss = 0.5 |generate(xi) - y|^2 + logdet through autograd (one adjoint sweep for both terms)
        XG.grad = None
        VG.grad = None
        v, ld = gg.generate_and_logdet(graph, (B, VG), XG)
        loss = 0.5 * torch.sum((v - y) ** 2) + ld
        loss.backward()
        return XG.grad, VG.grad.double()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        gx, gv = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    st = gc.last_status()

    # FP64 forward for the differences, and the FP64 adjoint beside the FP32 one
    P64, B64, V64 = gp.double(), B.double(), torch.as_tensor(vals, dtype=torch.float64, device=dev)
    y64, xi64 = y.double(), xi.double()

    def loss64(x, vv):
        v = gc.generate(P64, gi, gn, OF, B64, vv, x)
        return 0.5 * float(torch.sum((v - y64) ** 2)) + float(gc.generate_logdet(P64, gn, OF, B64, vv))

    v64 = gc.generate(P64, gi, gn, OF, B64, V64, xi64)
    gx64, gv64 = gc.generate_vjp(P64, gi, gn, OF, B64, V64, xi64, v64 - y64, 1.0)
    gx32, gv32 = gx.double(), gv.double()
    h = 1e-3
    res = {"xi": ([], []), "table": ([], []), "table_h1e-5": ([], [])}
    t0 = time.perf_counter()
    for i in range(n_dirs):
        if i % 2 == 0:
            ux = torch.as_tensor(rng.standard_normal(n), device=dev)
            ux /= torch.linalg.norm(ux)
            uv = torch.zeros_like(V64)
            runs = (("xi", h),)
        else:
            ux = torch.zeros_like(xi64)
            uv = torch.as_tensor(1e-3 * vals * rng.standard_normal(len(vals)), device=dev)
            runs = (("table", h), ("table_h1e-5", 1e-5))
        a32 = float(gx32 @ ux + gv32 @ uv)
        a64 = float(gx64 @ ux + gv64 @ uv)
        for name, hh in runs:
            fd = (loss64(xi64 + hh * ux, V64 + hh * uv) - loss64(xi64 - hh * ux, V64 - hh * uv)) / (2 * hh)
            scale = max(abs(fd), 1e-30)
            res[name][0].append(abs(a32 - fd) / scale)
            res[name][1].append(abs(a64 - fd) / scale)
    fd_s = time.perf_counter() - t0

    def stats(v):
        return {"max": float(np.max(v)), "median": float(np.median(v)), "count": len(v)} if v else None

    return {"workload": "differentiation: N = 4,194,304 uniform [0,1]^2, n0 = 256, k = 20, RBF scale 0.1, "
                        "r = 0 + 1,000 log bins on [1e-5, 1.5], jitter 1e-4; loss 0.5|generate(xi) - y|^2 + logdet",
            "value": n / (ms * 1e-3), "unit": "points/s", "ms_per_step": ms,
            "step": "FP32 loss = 0.5|generate(xi) - y|^2 + logdet and loss.backward() (graphgp_b200.generate_and_logdet: "
                    "forward values and logdet, one adjoint sweep; grad w.r.t. 4,194,304 xi and 1,001 table values)",
            "status_error": st["error"] if st else None, "fallback_points": st["fallback_count"] if st else None,
            "fd_directions": n_dirs, "fd_step": h,
            "fd_rel_err_fp32_adjoint": {k: stats(v[0]) for k, v in res.items()},
            "fd_rel_err_fp64_adjoint": {k: stats(v[1]) for k, v in res.items()},
            "grad_fp32_vs_fp64_rel": {"xi": float(torch.linalg.norm(gx32 - gx64) / torch.linalg.norm(gx64)),
                                      "table": float(torch.linalg.norm(gv32 - gv64) / torch.linalg.norm(gv64))},
            "fd_seconds": fd_s}


def largest(dev, n=1 << 28, steps=2):
    """The largest single instance: 2^28 points (largest_points), d = 3, n0 = 4096, k = 32, RBF scale 0.02 on
    r = 0 + 4,096 log bins over [1e-7, 4], jitter 1e-5. Times build_graph, generate and generate + adjoint, and
    checks the graph of the first 2^20 points bit for bit against the oracle's digests
    (tests/golden/largest_subset.json)."""
    import hashlib

    import torch

    from graphgp_b200 import extras
    from graphgp_b200 import graphgp_cuda as gc

    def digest(a):
        return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()

    out = {"workload": "largest instance: 2^28 points (64-cluster Gaussian mixture, sigma 10^U(-3,-1), plus 10% "
                       "uniform background in [-1,1]^3), d = 3, n0 = 4096, k = 32, RBF scale 0.02, r = 0 + 4,096 "
                       "log bins on [1e-7, 4], jitter 1e-5", "n_points": n}
    fx = json.loads(open(os.path.join(ROOT, "tests", "golden", "largest_subset.json")).read())
    sub = largest_points(fx["n"])
    gp, gi, gn, _, offs = gc.build_graph(torch.as_tensor(sub, device=dev), n0=fx["n0"], k=fx["k"], return_offsets=True)
    out["subset_bit_exact"] = bool(list(offs) == fx["offsets"]
                                   and digest(gi.cpu().numpy().astype(np.int32)) == fx["indices_sha256"]
                                   and digest(gn.cpu().numpy().astype(np.int32)) == fx["neighbors_sha256"]
                                   and digest(gp.cpu().numpy().astype(np.float32)) == fx["points_graph_sha256"])
    del gp, gi, gn
    t = time.perf_counter()
    pts = largest_points(n)
    out["host_generation_s"] = time.perf_counter() - t
    P = torch.as_tensor(pts, device=dev)
    del pts
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    gp, gi, gn, _, offs = gc.build_graph(P, n0=4096, k=32, return_offsets=True)
    e1.record()
    torch.cuda.synchronize()
    out["graph_build_ms"] = e0.elapsed_time(e1)
    out["batches"] = len(offs) - 1
    del P
    torch.cuda.empty_cache()
    OF = torch.as_tensor(offs, dtype=torch.int32, device=dev)
    B, V = extras.rbf_kernel(variance=1.0, scale=0.02, r_min=1e-7, r_max=4.0, n_bins=4097, jitter=1e-5, device=dev)
    xi = torch.randn(n, generator=torch.Generator(device=dev).manual_seed(3), device=dev)
    v = gc.generate(gp, gi, gn, OF, B, V, xi)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(steps):
        v = gc.generate(gp, gi, gn, OF, B, V, xi)
    e1.record()
    torch.cuda.synchronize()
    st = gc.last_status()
    out["generate_ms"] = e0.elapsed_time(e1) / steps
    out["generate_points_per_s"] = n / (out["generate_ms"] * 1e-3)
    out["generate_status"] = st
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(steps):
        v = gc.generate(gp, gi, gn, OF, B, V, xi)
        gx, gv = gc.generate_vjp(gp, gi, gn, OF, B, V, xi, v, 0.5, values=v)
    e1.record()
    torch.cuda.synchronize()
    out["generate_grad_ms"] = e0.elapsed_time(e1) / steps
    out["generate_grad_points_per_s"] = n / (out["generate_grad_ms"] * 1e-3)
    out["vjp_status"] = gc.last_status()
    out["finite"] = bool(torch.isfinite(v).all() and torch.isfinite(gx).all() and torch.isfinite(gv).all())
    out["peak_device_gb"] = torch.cuda.max_memory_allocated(dev) / 1e9
    return out


def serving(dev, n_requests):
    """The request stream (Poisson arrivals at 2000 req/s, uneven N, d, k, op mix 70/20/10) through the serving
    engine: 32 slots (one CUDA stream each), 64 GiB admission budget, latency = completion - arrival."""
    import torch

    from graphgp_b200 import serving as sv

    eng = sv.Engine(dev, slots=32, hbm_budget=64 << 30)
    # warm-up: one untimed pass over a different stream of the same distribution, so that the device memory
    # pool has grown to the stream's working set before the timed pass (a running server's steady state)
    eng.run(sv.synthetic_stream(n_requests=n_requests, rate=2000.0, seed=1), realtime=False)
    t = time.perf_counter()
    reqs = sv.synthetic_stream(n_requests=n_requests, rate=2000.0, seed=0)
    gen_s = time.perf_counter() - t
    torch.cuda.synchronize()
    res, summ = eng.run(reqs, realtime=True)
    bad = sum(1 for r in res if r.status and r.status.get("error"))
    pts = np.array([r.n for r in reqs])
    summ.update(warmup="one untimed pass over a 4096-request stream of the same distribution (seed 1)",
                workload="4096 requests, Poisson 2000 req/s, N lognormal(median 30000, log-sd 1) clipped to "
                         "[1e3, 1e6], d in {2,3}, k in {8,16,32}, n0 = max(k, min(256, N // 100)), RBF table per "
                         "request (scale U(0.05,0.5), r=0 + 999 log bins on [1e-4, 10]); op mix 70/20/10"
                if n_requests == 4096 else f"{n_requests} requests of the same distribution",
                total_points=int(pts.sum()), requests_with_error=bad, host_generation_s=gen_s,
                latency="completion - arrival, queueing included; includes graph build, H2D of points and "
                        "payload, the operation and D2H of the result")
    return summ


REFINE_KERNEL = "refine_quad2_kernel<float,16,3,false,kOpGenerate> (four lanes per point, generate)"
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the refinement kernel "
                  "(profiles/refine_quad_generate_c2.md, bytes per refined point), scaled to this launch's refined points")


def read_traffic(units):
    """DRAM bytes per refined point of the dominant kernel from the committed ncu summary, scaled to one
    launch; None when no capture has been summarised."""
    path = os.path.join(ROOT, "profiles", "refine_quad_generate_c2.md")
    try:
        for ln in open(path):
            if ln.startswith("dram_bytes_per_point:"):
                return float(ln.split(":")[1]) * units
    except OSError:
        pass
    return None


def comparisons(args, dev, gp, gi, gn, offs, OF, B, V, XI, pts, bins, vals, out32, ms32):
    """FP64 comparators on the full workload, and the FP32-vs-FP64 error of generate, inverse and log-determinant
    on the full workload and on a seed-matched 1M-point subset (its own graph). Errors are reported against FP64
    on the same inputs (the table rounded to FP32, as the FP32 kernels receive it) and, separately, against FP64
    with the unrounded table (which adds the effect of rounding the caller's table)."""
    import torch

    from graphgp_b200 import graphgp_cuda as gc

    res = {}
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    rel = lambda a, b: float(torch.linalg.vector_norm(a.double() - b) / torch.linalg.vector_norm(b))  # noqa: E731
    P64, X64 = gp.double(), XI.double()
    B64, V64 = B.double(), V.double()  # the FP32 inputs, held in FP64
    B64t, V64t = torch.as_tensor(bins, device=dev), torch.as_tensor(vals, device=dev)  # the unrounded table
    # (1) the same kernels instantiated in FP64
    out64 = gc.generate(P64, gi, gn, OF, B64, V64, X64)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(3):
        out64 = gc.generate(P64, gi, gn, OF, B64, V64, X64)
    e1.record()
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1) / 3
    res["fp64_same_kernels"] = {"ms_per_step": ms64, "speedup_fp32": ms64 / ms32}

    def errors(P32, I, NB, O, xs, v32, v64_same):
        """generate / inverse / logdet errors of the FP32 path against FP64 (same inputs, and unrounded table)."""
        Pd = P32.double()
        v64_tab = gc.generate(Pd, I, NB, O, B64t, V64t, xs.double())
        x32 = gc.generate_inv(P32, I, NB, O, B, V, v32)
        st_inv = gc.last_status()
        x64 = gc.generate_inv(Pd, I, NB, O, B64, V64, v32.double())
        x64t = gc.generate_inv(Pd, I, NB, O, B64t, V64t, v32.double())
        l32 = float(gc.generate_logdet(P32, NB, O, B, V))
        st_ld = gc.last_status()
        l64 = float(gc.generate_logdet(Pd, NB, O, B64, V64))
        l64t = float(gc.generate_logdet(Pd, NB, O, B64t, V64t))
        return {"generate": {"rel_err": rel(v32, v64_same), "rel_err_unrounded_table": rel(v32, v64_tab)},
                "inverse": {"rel_err": rel(x32, x64), "rel_err_unrounded_table": rel(x32, x64t),
                            "fp64_points": st_inv["fallback_count"]},
                "logdet": {"rel_err": abs(l32 - l64) / abs(l64), "rel_err_unrounded_table": abs(l32 - l64t) / abs(l64t),
                           "fp64_points": st_ld["fallback_count"], "value_fp32": l32, "value_fp64": l64}}

    res["errors_full"] = errors(gp, gi, gn, OF, XI, out32, out64)
    res["errors_full"]["note"] = ("FP32 path against the same kernels in FP64 on the same inputs; the inverse is of "
                                  "the FP32 generate output")
    del out64
    # (2) plain FP64-GPU form shaped like the reference's fast_jit path
    try:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ref = fp64_fastjit_generate(gp, gi, gn, offs, B64, V64, XI)
        torch.cuda.synchronize()
        msj = (time.perf_counter() - t0) * 1e3
        res["fp64_fastjit_form"] = {"ms_per_step": msj, "speedup_fp32": msj / ms32, "rel_err_fp32_vs_it": rel(out32, ref),
                                    "timing": "one call, wall clock with device synchronisation around it"}
        del ref
    except RuntimeError as exc:  # out of memory etc.
        res["fp64_fastjit_form"] = {"error": str(exc)[:200]}
    torch.cuda.empty_cache()
    # (3) a seed-matched 1M-point subset with its own graph
    m = min(1 << 20, len(pts))
    Ps = torch.as_tensor(pts[:m], device=dev)
    sp, si, sn, sd, so = gc.build_graph(Ps, n0=WORKLOAD["n0"], k=WORKLOAD["k"], return_offsets=True)
    SO = torch.as_tensor(so, dtype=torch.int32, device=dev)
    xs = XI[:m].contiguous()
    v32 = gc.generate(sp, si, sn, SO, B, V, xs)
    v64 = gc.generate(sp.double(), si, sn, SO, B64, V64, xs.double())
    res["subset_1m"] = errors(sp, si, sn, SO, xs, v32, v64)
    res["subset_1m"]["max_abs_err_generate"] = float((v32.double() - v64).abs().max())
    res["_subset"] = (sp, si, sn, so, xs, v32)
    return res


def cpu_baseline(subset, bins, vals, min_rows=100_000):
    """The NumPy FP64 oracle (reference refine.py:21-56 restated: dense root, per-point factorisation, batch scan)
    timed on this host, one core, on the first depth batches (at least min_rows refined points) of the 1M-point
    subset's graph. The same run checks the GPU's FP32 generate on those rows against it: rows in batches up to B
    depend only on earlier batches, so the oracle's values there are exact without the rest of the graph."""
    from oracle import refine as orf

    sp, si, sn, so, xs, v32 = subset
    n0 = WORKLOAD["n0"]
    cov = (np.asarray(bins, np.float32).astype(np.float64), np.asarray(vals, np.float32).astype(np.float64))
    nb = int(np.searchsorted(np.asarray(so), n0 + min_rows)) + 1
    nb = min(nb, len(so) - 1)
    end = int(so[nb])
    pts = sp[:end].cpu().numpy().astype(np.float64)
    idx = si.long().cpu().numpy()
    xg = xs.double().cpu().numpy()[idx]  # xi in graph order
    nbrs = sn[: end - n0].cpu().numpy()
    t0 = time.perf_counter()
    init = orf.generate_dense(pts[:n0], cov, xg[:n0])
    ref = orf.refine(pts, nbrs, tuple(int(x) for x in so[: nb + 1]), cov, init, xg[n0:end])
    dt = time.perf_counter() - t0
    gpu = v32.double().cpu().numpy()[idx][:end]
    err = float(np.linalg.norm(gpu - ref) / np.linalg.norm(ref))
    return {"value": (end - n0) / dt, "unit": "points/s", "cores": 1, "kind": "port",
            "sample": f"NumPy FP64 oracle generate (dense root n0 = {n0}, factorisation and batch scan) of the first "
                      f"{nb} depth batches ({end - n0} refined points) of the seed-matched 1M-point subset graph",
            "gpu_fp32_rel_err_vs_oracle": err, "rows_checked": end}


# ------------------------------------------------------------------------------------------------
# reference arm: the CPU restatement on all host cores
# ------------------------------------------------------------------------------------------------
def _ref_worker(payload):
    pts, nb, rows0, bins, vals, n0 = payload
    from oracle import refine as orf

    mv, sd = orf.factor_points(pts, nb, np.arange(n0 + rows0, n0 + rows0 + len(nb)), (bins, vals))
    return rows0, mv, sd


def run_reference(args, world, rank):
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle import graph as og

    w = WORKLOAD
    m = args.ref_sample
    pts = synth_points(w["n"], w["d"], w["seed"])[:m].astype(np.float64)
    bins, vals = table()
    g = og.build_graph(pts, n0=w["n0"], k=w["k"])  # untimed, like our arm's graph
    cores = os.cpu_count() or 1
    parts = np.array_split(np.arange(len(g.neighbors)), cores * 2)
    payloads = [(g.points, g.neighbors[p], int(p[0]), bins, vals, w["n0"]) for p in parts if len(p)]
    ctx = mp.get_context("spawn")
    xi = np.random.default_rng(w["seed"] + 1).standard_normal(len(g.points))
    m0 = len(g.neighbors)

    def generate_step(pool, pl):
        """The oracle's generate on the sample graph: dense root, per-point factorisation on every core, batch scan."""
        from oracle import refine as orf

        mv = np.empty((m0, w["k"]))
        sd = np.empty(m0)
        for rows0, a, b in pool.map(_ref_worker, pl):
            mv[rows0:rows0 + len(b)], sd[rows0:rows0 + len(b)] = a, b
        values = np.zeros(len(g.points))
        values[:w["n0"]] = orf.generate_dense(g.points[:w["n0"]], (bins, vals), xi[:w["n0"]])
        for b in range(1, len(g.offsets)):
            s0, e0 = g.offsets[b - 1], g.offsets[b]
            r = np.arange(s0 - w["n0"], e0 - w["n0"])
            values[s0:e0] = np.sum(mv[r] * values[g.neighbors[r]], axis=1) + sd[r] * xi[s0:e0]
        return m0

    with ctx.Pool(cores) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_worker, payloads[:cores])
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            done += generate_step(pool, payloads)
        dt = time.perf_counter() - t0
    val = done / dt
    print(json.dumps({
        "metric": METRIC, "value": val, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (same generator, first "
                                                       f"{m} points)",
        "config": {"workload": w["name"], "n_points": w["n"], "d": w["d"], "n0": w["n0"], "k": w["k"],
                   "sample_points": m},
        "impl": "reference",
        "cpu_baseline": {"value": val, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": f"generate of a {m}-point graph of the workload per step (NumPy FP64 oracle: dense "
                                   "root, per-point factorisation over a spawn pool of all cores, batch scan)"},
        "e2e": {"value": val, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=0, help="override the number of points (testing)")
    ap.add_argument("--quick", action="store_true", help="skip the FP64 comparators and CPU baseline")
    ap.add_argument("--ref-sample", type=int, default=200000)
    ap.add_argument("--serving-requests", type=int, default=4096, help="0 skips the serving stream")
    ap.add_argument("--largest", action=argparse.BooleanOptionalAction, default=True,
                    help="also run the 2^28-point largest instance (default; --no-largest skips it)")
    ap.add_argument("--only-differentiation", action="store_true",
                    help="run only the differentiation workload and print its object")
    ap.add_argument("--largest-n", type=int, default=1 << 28)
    ap.add_argument("--fd-directions", type=int, default=64,
                    help="finite-difference directions of the differentiation workload (0 skips it)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()
    if args.only_differentiation:
        import torch

        torch.cuda.set_device(local)
        print(json.dumps(differentiation(torch.device("cuda", local), n_dirs=args.fd_directions)), flush=True)
        return
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
