"""GPU parity of the refinement kernels (C-ABI via graphgp_b200.graphgp_cuda) against the FP64 oracle.

Tolerances: FP32 kernels vs the FP64 oracle at <= 1e-4 relative error (norm-wise over the output, the bar
the path is specified to); FP64 kernels at 1e-9 relative. The oracle runs on the inputs each kernel receives:
for FP32 kernels, the table rounded to FP32.
"""
import numpy as np
import pytest

from oracle import jax_random as jr
from oracle import graph as og
from oracle import refine as orf
from oracle import extras as ox

from conftest import rel_err
from helpers import as_inputs, oracle_graph, rbf_table, matern32_table

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL64 = 1e-9

CASES = [  # (n, d, n0, k, table)
    (3000, 2, 100, 10, "rbf"),
    (3000, 3, 256, 16, "matern"),
    (3000, 3, 128, 8, "rbf"),
    (3000, 2, 128, 20, "rbf"),
    (3000, 3, 128, 32, "rbf"),
    (3000, 2, 128, 5, "rbf"),     # padded to 8 (FP32), 16 (FP64)
    (3000, 3, 128, 12, "matern"),  # padded to 16
    (2500, 2, 128, 18, "matern"),  # padded to 20
    (2000, 3, 128, 24, "rbf"),     # padded to 32
]


def _table(name):
    return rbf_table() if name == "rbf" else matern32_table(cutoff=0.5)


def _t(x, dev, dtype=None):
    import torch

    t = torch.as_tensor(np.ascontiguousarray(x), device=dev)
    return t if dtype is None else t.to(dtype)


@pytest.mark.parametrize("n,d,n0,k,tab", CASES)
def test_refine_f32_vs_oracle(cuda_device, n, d, n0, k, tab):
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(_table(tab), np.float32)
    rng = np.random.default_rng(1)
    xi = rng.standard_normal(n)
    init = orf.generate_dense(g.points[:n0], (bins, vals), xi[:n0])
    ref = orf.refine(g.points, g.neighbors, g.offsets, (bins, vals), init, xi[n0:])
    f32 = torch.float32
    out = gc.refine(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device, f32),
                    _t(vals, cuda_device, f32), _t(init, cuda_device, f32), _t(xi[n0:], cuda_device, f32))
    st = gc.last_status()
    assert st["error"] == 0 and st["timeouts"] == 0
    assert rel_err(out.cpu().numpy(), ref) < TOL32

    # inverse: exact values in, xi out
    i0, xo = gc.refine_inv(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                           _t(bins, cuda_device, f32), _t(vals, cuda_device, f32), _t(ref, cuda_device, f32))
    ri0, rxi = orf.refine_inv(g.points, g.neighbors, g.offsets, (bins, vals), ref.astype(np.float32))
    assert np.array_equal(i0.cpu().numpy(), ref[:n0].astype(np.float32))
    assert rel_err(xo.cpu().numpy(), rxi) < TOL32  # points below the inverse's pivot threshold are FP64

    # logdet
    ld = gc.refine_logdet(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                          _t(bins, cuda_device, f32), _t(vals, cuda_device, f32))
    rld = orf.refine_logdet(g.points, g.neighbors, g.offsets, (bins, vals))
    assert abs(float(ld) - rld) / abs(rld) < TOL32


@pytest.mark.parametrize("n,d,n0,k,tab", [c for c in CASES if c[3] in (8, 10, 16, 20, 5, 12, 18)])
def test_refine_f64_vs_oracle(cuda_device, n, d, n0, k, tab):
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = _table(tab)
    rng = np.random.default_rng(2)
    xi = rng.standard_normal(n)
    p64 = g.points.astype(np.float64)
    init = orf.generate_dense(p64[:n0], (bins, vals), xi[:n0])
    ref = orf.refine(p64, g.neighbors, g.offsets, (bins, vals), init, xi[n0:])
    out = gc.refine(_t(p64, cuda_device), _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device),
                    _t(vals, cuda_device), _t(init, cuda_device), _t(xi[n0:], cuda_device))
    assert rel_err(out.cpu().numpy(), ref) < TOL64
    ld = gc.refine_logdet(_t(p64, cuda_device), _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device),
                          _t(vals, cuda_device))
    rld = orf.refine_logdet(p64, g.neighbors, g.offsets, (bins, vals))
    assert abs(float(ld) - rld) / abs(rld) < TOL64


@pytest.mark.parametrize("d,k", [(4, 6), (3, 40), (1, 4)])
def test_generic_path_vs_oracle(cuda_device, d, k):
    """Shapes outside the register-resident kernels take the block-per-point FP64 path."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, n0 = 1500, max(64, k)
    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(rbf_table(scale=0.8), np.float32)
    xi = np.random.default_rng(3).standard_normal(n)
    init = orf.generate_dense(g.points[:n0], (bins, vals), xi[:n0])
    ref = orf.refine(g.points, g.neighbors, g.offsets, (bins, vals), init, xi[n0:])
    f32 = torch.float32
    out = gc.refine(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device, f32),
                    _t(vals, cuda_device, f32), _t(init, cuda_device, f32), _t(xi[n0:], cuda_device, f32))
    assert rel_err(out.cpu().numpy(), ref) < TOL32
    ld = gc.refine_logdet(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                          _t(bins, cuda_device, f32), _t(vals, cuda_device, f32))
    rld = orf.refine_logdet(g.points, g.neighbors, g.offsets, (bins, vals))
    assert abs(float(ld) - rld) / abs(rld) < TOL32


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_generate_whole_vs_oracle(cuda_device, dtype):
    """generate / generate_inv / generate_logdet with the indices permutation, dense root in FP64."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, d, n0, k = 4000, 2, 300, 10
    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(rbf_table(), getattr(np, dtype))
    xi = np.random.default_rng(4).standard_normal(n)
    ref = orf.generate(g, (bins, vals), xi)
    tdt = getattr(torch, dtype)
    args = (_t(g.points, cuda_device, tdt), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
            _t(bins, cuda_device, tdt), _t(vals, cuda_device, tdt))
    out = gc.generate(*args, _t(xi, cuda_device, tdt)).cpu().numpy()
    tol = TOL32 if dtype == "float32" else TOL64
    assert rel_err(out, ref) < tol
    back = gc.generate_inv(*args, _t(ref, cuda_device, tdt)).cpu().numpy()
    assert rel_err(back, orf.generate_inv(g, (bins, vals), ref.astype(dtype))) < tol
    ld = float(gc.generate_logdet(args[0], args[2], args[3], args[4], args[5]))
    rld = orf.generate_logdet(g, (bins, vals))
    assert abs(ld - rld) / abs(rld) < tol


def test_dense_root_vs_oracle(cuda_device):
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    rng = np.random.default_rng(5)
    for n0 in (1, 37, 63, 64, 65, 128, 129, 200, 1030):  # ragged and whole 64-row tiles
        pts = rng.standard_normal((n0, 3))
        bins, vals = ox.matern_kernel(p=1, variance=1.0, cutoff=1.0, r_min=1e-4, r_max=20, n_bins=1000, jitter=1e-5)
        tb, tv, tp = _t(bins, cuda_device), _t(vals, cuda_device), _t(pts, cuda_device)
        x = rng.standard_normal(n0)
        gen = gc.dense("generate", tp, tb, tv, _t(x, cuda_device)).cpu().numpy()
        assert rel_err(gen, orf.generate_dense(pts, (bins, vals), x)) < 1e-11
        inv = gc.dense("inverse", tp, tb, tv, _t(gen, cuda_device)).cpu().numpy()
        assert rel_err(inv, x) < 1e-8
        ld = float(gc.dense("logdet", tp, tb, tv))
        rld = orf.generate_dense_logdet(pts, (bins, vals))
        assert abs(ld - rld) <= 1e-10 * max(1.0, abs(rld))


def test_reference_logdet_golden(cuda_device):
    """Reference tests/test_refine.py:29-43: jr.key(137) points (1000, 3), n0=100, k=10, Matern p=0 table;
    generate_logdet == -600.36165088 and dense logdet of all points == -610.90538067 (rtol 1e-8), here in FP64
    on the GPU with the graph from the oracle."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = jr.normal(jr.key(137), (1000, 3))
    g = og.build_graph(pts, n0=100, k=10)
    assert abs(g.points[0, 0] - (-1.95624711)) < 1e-8 * 1.96
    bins, vals = ox.matern_kernel(p=0, variance=1.0, cutoff=1.0, r_min=1e-4, r_max=10, n_bins=1000, jitter=1e-5)
    ld = float(gc.generate_logdet(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                                  _t(bins, cuda_device), _t(vals, cuda_device)))
    assert abs(ld - (-600.36165088)) <= 1e-8 * 600.36165088
    dl = float(gc.dense("logdet", _t(g.points, cuda_device), _t(bins, cuda_device), _t(vals, cuda_device)))
    assert abs(dl - (-610.90538067)) <= 1e-8 * 610.90538067


def test_wait_probe_times_out(cuda_device):
    """A bounded device wait on a flag nothing sets returns GGP_ERR_TIMEOUT and leaves the context usable."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    assert gc.wait_probe(2_000_000) == 3
    x = torch.ones(4, device=cuda_device)
    assert float(x.sum()) == 4.0


def test_invalid_graph_reports_not_hangs(cuda_device):
    """A neighbour inside its own batch violates check_graph (reference graph.py:62-70): the kernel reports
    GGP_ERR_INVALID and yields NaN instead of waiting on a later ticket."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(1000, 2, 64, 8)
    nb = g.neighbors.copy()
    nb[0, 0] = g.offsets[0]  # first refined point depends on itself: same batch
    bins, vals = rbf_table()
    f32 = torch.float32
    out = gc.refine(_t(g.points, cuda_device), _t(nb, cuda_device), g.offsets, _t(bins, cuda_device, f32),
                    _t(vals, cuda_device, f32), torch.zeros(64, device=cuda_device),
                    torch.zeros(1000 - 64, device=cuda_device), timeout_ns=50_000_000)
    st = gc.last_status()
    assert st["error"] == 1
    assert torch.isnan(out[g.offsets[0]]).item()


@pytest.mark.parametrize("k,d", [(32, 3), (24, 2)])
def test_inverse_logdet_list_pass_k32(cuda_device, k, d):
    """k above the quad list kernel's sizes: the FP32 first pass lists its points below tau and the
    warp-per-point FP64 pass finishes them; inverse and logdet stay within the FP32 bar of the FP64 oracle."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, n0 = 2500, 128
    pts, g = oracle_graph(n, d, n0, k, seed=11)
    bins, vals = as_inputs(rbf_table(scale=0.5), np.float32)
    f32 = torch.float32
    args = (_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device, f32),
            _t(vals, cuda_device, f32))
    v = np.random.default_rng(2).standard_normal(n).astype(np.float32)
    i0, xi = gc.refine_inv(*args, _t(v, cuda_device, f32))
    listed = int(gc._tls.last_ws[:64].view(torch.int32)[7].item())
    assert listed > 0  # the smooth table puts points below the inverse threshold
    ri0, rxi = orf.refine_inv(g.points, g.neighbors, g.offsets, (bins, vals), v)
    assert rel_err(xi.cpu().numpy(), rxi) < TOL32
    ld = float(gc.refine_logdet(*args))
    rld = orf.refine_logdet(g.points, g.neighbors, g.offsets, (bins, vals))
    assert abs(ld - rld) / abs(rld) < TOL32


@pytest.mark.parametrize("tab,expect_all", [("rbf", 1), ("matern", 0)])
def test_inverse_sampling_decides_fp64_share(cuda_device, tab, expect_all):
    """The FP32 inverse samples every 32nd chunk first: with a smooth table most rows fall below the threshold and
    every row is finished in FP64 (the FP32 pass is skipped); with a rough one the ordinary FP32 pass and row list
    run. Both stay within the FP32 bar of the FP64 oracle."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, d, n0, k = 4000, 2, 128, 10
    pts, g = oracle_graph(n, d, n0, k, seed=3)
    bins, vals = as_inputs(_table(tab), np.float32)
    f32 = torch.float32
    v = np.random.default_rng(9).standard_normal(n).astype(np.float32)
    i0, xi = gc.refine_inv(_t(g.points, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                           _t(bins, cuda_device, f32), _t(vals, cuda_device, f32), _t(v, cuda_device, f32))
    st = gc._tls.last_ws[:64].view(torch.int32).cpu().numpy()
    assert int(st[12]) == expect_all  # DeviceStatus.all_fp64
    if expect_all:
        assert int(st[7]) == n - n0  # every row listed
    ri0, rxi = orf.refine_inv(g.points, g.neighbors, g.offsets, (bins, vals), v)
    assert rel_err(xi.cpu().numpy(), rxi) < TOL32


@pytest.mark.parametrize("d,k", [(2, 10), (3, 16), (3, 32), (4, 8)])
def test_generate_and_logdet_one_pass(cuda_device, d, k):
    """generate_and_logdet (FP32, one pass: the dense root and the refinement kernel also sum the log-determinant)
    gives generate's values bit for bit and generate_logdet's log-determinant to FP64 rounding, for the
    one-thread-per-point (k <= 10), four-lane (k 16, 32) and generic (d = 4) kernels."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, n0 = 3000, 200
    pts, g = oracle_graph(n, d, n0, k, seed=13)
    bins, vals = as_inputs(rbf_table(), np.float32)
    f32 = torch.float32
    args = (_t(g.points, cuda_device), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
            _t(bins, cuda_device, f32), _t(vals, cuda_device, f32))
    xi = _t(np.random.default_rng(1).standard_normal(n).astype(np.float32), cuda_device)
    v, ld = gc.generate_and_logdet(*args, xi)
    assert torch.equal(v, gc.generate(*args, xi))
    ref = float(gc.generate_logdet(args[0], args[2], args[3], args[4], args[5]))
    assert abs(float(ld) - ref) <= 1e-9 * abs(ref)
    rld = orf.generate_logdet(g, (bins, vals))
    assert abs(float(ld) - rld) / abs(rld) < TOL32
