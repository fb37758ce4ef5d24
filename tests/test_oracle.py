"""The oracle against the reference's own tests (CPU only).

Each test restates one test of stanford-ism/graphgp (cited) on the NumPy oracle: known answers, the
RNG-bound goldens (inputs regenerated with the threefry restatement, checked by the reference's RNG
sentinels), and the property tests (brute-force k-NN, inverse round trip, two-implementation agreement,
dense limit).
"""
import numpy as np
import pytest

from oracle import extras as ox
from oracle import graph as og
from oracle import jax_random as jr
from oracle import refine as orf
from oracle import tree as ot

KEY = jr.key(137)


def test_rng_sentinel():
    """tests/test_tree.py:29 / test_graph.py:23: points[0, 0] == -0.61777326 for jr.normal(key(137), ...)."""
    pts = jr.normal(KEY, (100000, 3))
    assert abs(pts[0, 0] - (-0.61777326)) <= 1e-8 * 0.61777326
    # the partitionable counter layout makes a smaller draw a prefix of a larger one
    assert np.array_equal(jr.normal(KEY, (1000, 3)), pts[:1000])


def test_build_tree_simple():
    """tests/test_tree.py:19-24."""
    p, s, i = ot.build_tree(np.arange(1, 11, dtype=np.float64)[:, None])
    assert np.array_equal(p[:, 0], [6, 3, 9, 2, 8, 5, 10, 1, 7, 4])
    assert np.array_equal(s, np.zeros(10))
    assert np.array_equal(i, [5, 2, 8, 1, 7, 4, 9, 0, 6, 3])


def test_build_tree_random_golden():
    """tests/test_tree.py:27-32."""
    p, s, i = ot.build_tree(jr.normal(KEY, (100000, 3)))
    assert np.array_equal(s[1000:1005], [2, 0, 0, 1, 1])
    assert i[-1] == 59735


def test_build_tree_shapes():
    """tests/test_tree.py:35-41."""
    for d in (2, 6):
        p, s, i = ot.build_tree(jr.normal(KEY, (1000, d)))
        assert p.shape == (1000, d) and s.shape == (1000,) and i.shape == (1000,)


def test_query_preceding_brute_force():
    """tests/test_tree.py:44-59."""
    p, s, _ = ot.build_tree(jr.normal(KEY, (1000, 3)))
    nb = ot.query_preceding_neighbors(p, s, n0=30, k=30)
    dist = np.linalg.norm(p[:, None, :] - p[None, :, :], axis=-1)
    ii, jj = np.indices(dist.shape)
    dist[ii <= jj] = np.inf
    assert np.array_equal(nb, np.argsort(dist, axis=-1, kind="stable")[30:, :30])


def test_tree_index_arithmetic():
    """tree.py:187-208: children of j are j + 2^l and j + 2^(l+1); parent inverts both; root's parent -1."""
    j = np.arange(0, 5000)
    assert np.array_equal(ot.compute_parent(ot.compute_left(j)), j)
    assert np.array_equal(ot.compute_parent(ot.compute_right(j)), j)
    assert ot.compute_parent(np.array([0]))[0] == -1
    assert list(ot.compute_left(np.array([0, 1, 2]))) == [1, 3, 4]
    assert list(ot.compute_right(np.array([0, 1, 2]))) == [2, 5, 6]


def test_graph_random_golden():
    """tests/test_graph.py:14-27."""
    g = og.build_graph(jr.normal(KEY, (100000, 3)), n0=1000, k=10)
    assert len(g.offsets) == 61 and g.offsets[1] == 1115
    assert g.neighbors[0, 0] == 488
    assert abs(g.points[0, 0] - (-1.38417124)) <= 1e-8 * 1.38417124
    og.check_graph(g)


def test_graph_shapes():
    """tests/test_graph.py:30-37."""
    g = og.build_graph(jr.normal(KEY, (5000, 6)), n0=500, k=15)
    assert g.points.shape == (5000, 6) and g.neighbors.shape == (4500, 15) and g.indices.shape == (5000,)
    assert g.offsets[0] == 500 and g.offsets[-1] == 5000


def test_compute_depths():
    """tests/test_graph.py:40-52."""
    nb = np.array([[0, 1, 2], [0, 1, 2], [1, 3, 4], [2, 4, 5]])
    assert np.array_equal(og.compute_depths(nb, n0=3), [0, 0, 0, 1, 1, 2, 3])


def test_order_by_depth():
    """tests/test_graph.py:55-82."""
    pts = np.arange(6, dtype=np.float64)[:, None]
    nb = np.array([[0, 1], [1, 2], [2, 3], [0, 1]])
    p, i, n, d = og.order_by_depth(pts, np.arange(6), nb, np.array([0, 0, 1, 2, 3, 1]))
    assert np.array_equal(p[:, 0], [0, 1, 2, 5, 3, 4]) and np.array_equal(i, [0, 1, 2, 5, 3, 4])
    assert np.array_equal(n, [[0, 1], [0, 1], [1, 2], [2, 4]]) and np.array_equal(d, [0, 0, 1, 1, 2, 3])


def test_check_graph_rejects_same_batch():
    g = og.build_graph(np.random.default_rng(0).standard_normal((500, 2)), n0=20, k=5)
    bad = og.Graph(g.points, g.neighbors.copy(), g.offsets, g.indices)
    bad.neighbors[0, 0] = g.offsets[0]
    with pytest.raises(AssertionError):
        og.check_graph(bad)


@pytest.fixture(scope="module")
def refine_setup():
    """tests/test_refine.py:15-26."""
    g = og.build_graph(jr.normal(KEY, (1000, 3)), n0=100, k=10)
    cov = ox.matern_kernel(p=0, variance=1.0, cutoff=1.0, r_min=1e-4, r_max=10, n_bins=1000, jitter=1e-5)
    return g, cov


def test_logdet_random_golden(refine_setup):
    """tests/test_refine.py:29-43."""
    g, cov = refine_setup
    assert abs(g.points[0, 0] - (-1.95624711)) <= 1e-8 * 1.95624711
    assert abs(orf.generate_logdet(g, cov) - (-600.36165088)) <= 1e-8 * 600.36165088
    assert abs(orf.generate_dense_logdet(g.points, cov) - (-610.90538067)) <= 1e-8 * 610.90538067


def test_inverse_round_trip(refine_setup):
    """tests/test_refine.py:46-54 (rtol 1e-12)."""
    g, cov = refine_setup
    xi = np.random.default_rng(0).standard_normal(1000)
    v = orf.generate(g, cov, xi)
    v2 = orf.generate(g, cov, orf.generate_inv(g, cov, v))
    assert np.allclose(v, v2, rtol=1e-12)


def test_fast_jit_matches_simple(refine_setup):
    """tests/test_refine.py:57-63 (rtol 1e-12)."""
    g, cov = refine_setup
    xi = np.random.default_rng(1).standard_normal(1000)
    assert np.allclose(orf.generate(g, cov, xi), orf.generate(g, cov, xi, mode="simple"), rtol=1e-12)


def test_approaches_dense():
    """tests/test_refine.py:66-80: k = n0 = 200 of 1000 points; values and J J^T close to dense (atol 0.02)."""
    g = og.build_graph(jr.normal(KEY, (1000, 3)), n0=200, k=200)
    g = og.Graph(g.points, g.neighbors, g.offsets)
    cov = ox.matern_kernel(p=0, variance=1.0, cutoff=1.0, r_min=1e-4, r_max=10, n_bins=1000, jitter=1e-5)
    xi = jr.normal(KEY, (1000,))  # the reference draws xi with the same key (test_refine.py:154)
    assert np.allclose(orf.generate_dense(g.points, cov, xi), orf.generate(g, cov, xi), atol=0.02)
    # generate is linear in xi: J = generate applied to the identity, batch by batch
    n0 = 200
    mv, sd = orf.factor_all(g.points, g.neighbors, cov, n0)
    J = np.zeros((1000, 1000))
    K0 = orf.compute_cov_matrix(cov, g.points[:n0], g.points[:n0])
    J[:n0, :n0] = np.linalg.cholesky(K0)
    for b in range(1, len(g.offsets)):
        s, e = g.offsets[b - 1], g.offsets[b]
        rows = np.arange(s - n0, e - n0)
        J[s:e] = np.einsum("rk,rkj->rj", mv[rows], J[g.neighbors[rows]])
        J[s:e, s:e] += np.diag(sd[rows])
    dense = orf.compute_cov_matrix(cov, g.points, g.points)
    assert np.allclose(J @ J.T, dense, atol=0.02)


def test_interp_matches_numpy():
    """cov_lookup restates jnp.interp: equal to np.interp inside the table and clamped outside."""
    bins, vals = ox.rbf_kernel(variance=1.0, scale=0.3, r_min=1e-4, r_max=10, n_bins=1001, jitter=1e-4)
    r = np.concatenate([[0.0, 1e-5, 1e-4, 10.0, 11.0], np.random.default_rng(3).uniform(0, 12, 1000)])
    assert np.allclose(orf.cov_lookup(r, bins, vals), np.interp(r, bins, vals), rtol=1e-12, atol=1e-15)
