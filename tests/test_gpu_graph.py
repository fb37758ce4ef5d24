"""GPU parity of the graph build (k-d tree, preceding k-NN, depths, ordering, offsets) against the oracle.

Everything here is integer / ordering work, so the bar is bit-exact equality, including ties (duplicate
coordinates) and the reference's own golden values (tests/test_tree.py, tests/test_graph.py).
"""
import numpy as np
import pytest

from oracle import graph as og
from oracle import jax_random as jr
from oracle import tree as ot

pytestmark = pytest.mark.gpu


def _t(x, dev):
    import torch

    return torch.as_tensor(np.ascontiguousarray(x), device=dev)


def _np(t):
    return t.cpu().numpy()


def test_build_tree_simple(cuda_device):
    """Reference tests/test_tree.py:19-24."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.arange(1, 11, dtype=np.float32)[:, None]
    p, s, i = gc.build_tree(_t(pts, cuda_device))
    assert np.array_equal(_np(p)[:, 0], [6, 3, 9, 2, 8, 5, 10, 1, 7, 4])
    assert np.array_equal(_np(s), np.zeros(10))
    assert np.array_equal(_np(i), [5, 2, 8, 1, 7, 4, 9, 0, 6, 3])


def test_build_tree_reference_golden(cuda_device):
    """Reference tests/test_tree.py:27-32 (jr.key(137), 100000 x 3, float64)."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = jr.normal(jr.key(137), (100000, 3))
    p, s, i = gc.build_tree(_t(pts, cuda_device))
    s, i = _np(s), _np(i)
    assert np.array_equal(s[1000:1005], [2, 0, 0, 1, 1])
    assert i[-1] == 59735
    rp, rs, ri = ot.build_tree(pts)
    assert np.array_equal(_np(p), rp) and np.array_equal(s, rs) and np.array_equal(i, ri)


@pytest.mark.parametrize("n,d", [(1, 2), (2, 3), (3, 1), (31, 2), (32, 3), (33, 2), (1000, 3), (4097, 2), (5000, 6),
                                 (70000, 3), (300001, 2)])
def test_build_tree_vs_oracle(cuda_device, n, d):
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.random.default_rng(n + d).standard_normal((n, d)).astype(np.float32)
    p, s, i = gc.build_tree(_t(pts, cuda_device))
    rp, rs, ri = ot.build_tree(pts)
    assert np.array_equal(_np(i), ri)
    assert np.array_equal(_np(s), rs)
    assert np.array_equal(_np(p), rp)


@pytest.mark.parametrize("kind", ["lattice", "rounded", "duplicates"])
def test_build_tree_ties_vs_oracle(cuda_device, kind):
    """Duplicate coordinates: the median falls on ties, resolved by ancestor coordinates then index."""
    from graphgp_b200 import graphgp_cuda as gc

    rng = np.random.default_rng(7)
    if kind == "lattice":
        g = np.stack(np.meshgrid(np.arange(96), np.arange(80)), -1).reshape(-1, 2)
        pts = g[rng.permutation(len(g))].astype(np.float32)
    elif kind == "rounded":
        pts = np.round(rng.standard_normal((50000, 3)) * 8) / 8
        pts = pts.astype(np.float32)
    else:
        base = rng.standard_normal((3000, 3)).astype(np.float32)
        pts = base[rng.integers(0, 3000, 20000)]
    p, s, i = gc.build_tree(_t(pts, cuda_device))
    rp, rs, ri = ot.build_tree(pts)
    assert np.array_equal(_np(i), ri)
    assert np.array_equal(_np(s), rs)


@pytest.mark.parametrize("n,d,n0,k", [(20000, 2, 100, 10), (20000, 3, 64, 16), (10000, 3, 64, 32), (3000, 2, 64, 40),
                                      (4000, 6, 50, 15), (3000, 1, 20, 8)])
def test_query_preceding_vs_oracle(cuda_device, n, d, n0, k):
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.random.default_rng(11 * n + d).standard_normal((n, d)).astype(np.float32)
    rp, rs, ri = ot.build_tree(pts)
    nb = _np(gc.query_preceding_neighbors(_t(rp, cuda_device), _t(rs, cuda_device), n0=n0, k=k))
    ref = ot.query_preceding_neighbors(rp, rs, n0=n0, k=k)
    assert np.array_equal(nb, ref)


def test_query_preceding_brute_force(cuda_device):
    """Reference tests/test_tree.py:44-59: k = n0 = 30 neighbours equal the masked argsort of distances."""
    from graphgp_b200 import graphgp_cuda as gc

    pts0 = jr.normal(jr.key(137), (1000, 3))
    p, s, _ = gc.build_tree(_t(pts0, cuda_device))
    nb = _np(gc.query_preceding_neighbors(p, s, n0=30, k=30))
    pts = _np(p)
    dist = np.linalg.norm(pts[:, None, :] - pts[None, :, :], axis=-1)
    ii, jj = np.indices(dist.shape)
    dist[ii <= jj] = np.inf
    true = np.argsort(dist, axis=-1, kind="stable")[30:, :30]
    assert np.array_equal(nb, true)


@pytest.mark.parametrize("k,small_max", [(12, False), (32, True), (16, True)])
def test_query_neighbors_arbitrary(cuda_device, k, small_max):
    """Arbitrary query ids and per-query search limits. ``small_max`` adds limits of 0 (only the root is visited,
    as in the reference's traversal) and below k (unfilled slots, ordered against the last point like the
    reference)."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.random.default_rng(3).standard_normal((5000, 3)).astype(np.float32)
    rp, rs, _ = ot.build_tree(pts)
    rng = np.random.default_rng(4 + k)
    q = rng.integers(0, 5000, 700)
    m = np.maximum(rng.integers(0, 5000, 700), k)
    if small_max:
        m[:60] = rng.integers(0, 2 * k, 60)
        m[:5] = 0
    out = _np(gc.query_neighbors(_t(rp, cuda_device), _t(rs, cuda_device), _t(q.astype(np.int32), cuda_device),
                                 _t(m.astype(np.int32), cuda_device), k=k))
    ref = ot.query_neighbors(rp, rs, q, m, k=k)
    assert np.array_equal(out, ref)


def test_compute_depths_known_answer(cuda_device):
    """Reference tests/test_graph.py:40-52."""
    from graphgp_b200 import graphgp_cuda as gc

    nb = np.array([[0, 1, 2], [0, 1, 2], [1, 3, 4], [2, 4, 5]], dtype=np.int32)
    out = _np(gc.compute_depths_parallel(_t(nb, cuda_device), n0=3))
    assert np.array_equal(out, [0, 0, 0, 1, 1, 2, 3])


def test_order_by_depth_known_answer(cuda_device):
    """Reference tests/test_graph.py:55-82."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.arange(6, dtype=np.float32)[:, None]
    idx = np.arange(6, dtype=np.int32)
    nb = np.array([[0, 1], [1, 2], [2, 3], [0, 1]], dtype=np.int32)
    dep = np.array([0, 0, 1, 2, 3, 1], dtype=np.int32)
    p, i, n, d = gc.order_by_depth(*(_t(x, cuda_device) for x in (pts, idx, nb, dep)))
    assert np.array_equal(_np(p)[:, 0], [0, 1, 2, 5, 3, 4])
    assert np.array_equal(_np(i), [0, 1, 2, 5, 3, 4])
    assert np.array_equal(_np(n), [[0, 1], [0, 1], [1, 2], [2, 4]])
    assert np.array_equal(_np(d), [0, 0, 1, 1, 2, 3])


@pytest.mark.parametrize("n,d,n0,k", [(30000, 2, 100, 10), (30000, 3, 1024, 16), (8000, 3, 64, 32)])
def test_depths_order_vs_oracle(cuda_device, n, d, n0, k):
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.random.default_rng(n + k).standard_normal((n, d)).astype(np.float32)
    rp, rs, ri = ot.build_tree(pts)
    nb = ot.query_preceding_neighbors(rp, rs, n0=n0, k=k)
    dep = _np(gc.compute_depths_parallel(_t(nb.astype(np.int32), cuda_device), n0=n0))
    rdep = og.compute_depths(nb, n0=n0)
    assert np.array_equal(dep, rdep)
    p, i, nn, dd, offs = gc.order_by_depth(_t(rp, cuda_device), _t(ri.astype(np.int32), cuda_device),
                                           _t(nb.astype(np.int32), cuda_device), _t(dep, cuda_device),
                                           return_offsets=True)
    rp2, ri2, rn2, rd2 = og.order_by_depth(rp, ri, nb, rdep)
    assert np.array_equal(_np(p), rp2) and np.array_equal(_np(i), ri2)
    assert np.array_equal(_np(nn), rn2) and np.array_equal(_np(dd), rd2)
    assert offs == og.compute_offsets(rd2)


def test_build_graph_reference_golden(cuda_device):
    """Reference tests/test_graph.py:14-27 (jr.key(137), 100000 x 3, n0=1000, k=10, float64)."""
    from graphgp_b200 import graphgp_cuda as gc

    pts = jr.normal(jr.key(137), (100000, 3))
    p, i, nb, dep, offs = gc.build_graph(_t(pts, cuda_device), n0=1000, k=10, return_offsets=True)
    assert len(offs) == 61 and offs[1] == 1115
    assert _np(nb)[0, 0] == 488
    assert abs(_np(p)[0, 0] - (-1.38417124)) <= 1e-8 * 1.38417124
    g = og.build_graph(pts, n0=1000, k=10)
    assert np.array_equal(_np(p), g.points) and np.array_equal(_np(i), g.indices)
    assert np.array_equal(_np(nb), g.neighbors) and offs == g.offsets


@pytest.mark.parametrize("n,d,n0,k", [(5000, 6, 500, 15), (100000, 2, 100, 10), (60000, 3, 1024, 16)])
def test_build_graph_vs_oracle(cuda_device, n, d, n0, k):
    from graphgp_b200 import graphgp_cuda as gc

    pts = np.random.default_rng(99).standard_normal((n, d)).astype(np.float32)
    p, i, nb, dep, offs = gc.build_graph(_t(pts, cuda_device), n0=n0, k=k, return_offsets=True)
    g = og.build_graph(pts, n0=n0, k=k)
    assert offs[0] == n0 and offs[-1] == n
    assert np.array_equal(_np(i), g.indices)
    assert np.array_equal(_np(p), g.points)
    assert np.array_equal(_np(nb), g.neighbors)
    assert offs == g.offsets
    og.check_graph(og.Graph(_np(p), _np(nb), offs, _np(i)))


def test_largest_instance_subset_bit_exact(cuda_device):
    """The largest-instance workload's parity subset (its first 2^20 points: 64-cluster Gaussian mixture plus
    uniform background, d = 3, n0 = 4096, k = 32): the GPU graph (indices, neighbours, ordered points,
    offsets) equals the oracle's bit for bit, compared through the SHA-256 digests that
    tests/golden/make_largest_subset.py recorded from the oracle."""
    import hashlib
    import json
    from pathlib import Path

    import torch

    from bench import largest_points
    from graphgp_b200 import graphgp_cuda as gc

    fx = json.loads((Path(__file__).parent / "golden" / "largest_subset.json").read_text())

    def digest(a):
        return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()

    pts = largest_points(fx["n"])
    assert digest(pts) == fx["points_sha256"]
    gp, gi, gn, _, offs = gc.build_graph(torch.as_tensor(pts, device=cuda_device), n0=fx["n0"], k=fx["k"],
                                         return_offsets=True)
    assert list(offs) == fx["offsets"]
    assert digest(gi.cpu().numpy().astype(np.int32)) == fx["indices_sha256"]
    assert digest(gn.cpu().numpy().astype(np.int32)) == fx["neighbors_sha256"]
    assert digest(gp.cpu().numpy().astype(np.float32)) == fx["points_graph_sha256"]
