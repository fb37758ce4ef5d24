"""Edge cases of the device path against the oracle: every point dense (n = n0, no refined rows), k = 1 with
n0 = 1, one dimension, duplicated points (exact ties) and tiny graphs. The graph must be bit-exact; generate,
generate_inv and generate_logdet in FP64 within 1e-9 relative."""
import numpy as np
import pytest
import torch

import graphgp_b200 as gp
from oracle import graph as og
from oracle import refine as orf

from conftest import rel_err
from helpers import rbf_table

pytestmark = pytest.mark.gpu


def _check(cuda_device, pts, n0, k):
    bins, vals = rbf_table(scale=0.5)
    g = og.build_graph(pts, n0=n0, k=k)
    graph = gp.build_graph(torch.as_tensor(pts, device=cuda_device), n0=n0, k=k)
    assert graph.offsets == tuple(g.offsets)
    assert np.array_equal(graph.indices.cpu().numpy(), g.indices)
    assert np.array_equal(graph.neighbors.cpu().numpy().reshape(g.neighbors.shape), g.neighbors)
    if len(g.neighbors):
        gp.check_graph(graph)
    g64 = gp.Graph(graph.points.double(), graph.neighbors, graph.offsets, graph.indices)
    cov = (torch.as_tensor(bins, device=cuda_device), torch.as_tensor(vals, device=cuda_device))
    xi = np.random.default_rng(len(pts)).standard_normal(len(pts))
    v = gp.generate(g64, cov, torch.as_tensor(xi, device=cuda_device)).cpu().numpy()
    ref = orf.generate(g, (bins, vals), xi)
    assert np.all(np.isfinite(v))
    assert rel_err(v, ref) < 1e-9
    x2 = gp.generate_inv(g64, cov, torch.as_tensor(ref, device=cuda_device)).cpu().numpy()
    assert rel_err(x2, orf.generate_inv(g, (bins, vals), ref)) < 1e-9
    ld = float(gp.generate_logdet(g64, cov))
    rld = orf.generate_logdet(g, (bins, vals))
    assert abs(ld - rld) <= 1e-9 * max(1.0, abs(rld))


def test_all_points_dense(cuda_device):
    pts = np.random.default_rng(1).standard_normal((200, 2)).astype(np.float32)
    _check(cuda_device, pts, n0=200, k=8)


def test_k1_n0_1(cuda_device):
    pts = np.random.default_rng(2).standard_normal((500, 2)).astype(np.float32)
    _check(cuda_device, pts, n0=1, k=1)


def test_one_dimension(cuda_device):
    pts = np.random.default_rng(3).standard_normal((800, 1)).astype(np.float32)
    _check(cuda_device, pts, n0=16, k=4)


def test_duplicated_points(cuda_device):
    """Exact duplicates: the graph is bit-exact (the ties), but a point whose neighbourhood holds its own
    duplicate has an exactly singular joint covariance (r = 0 gives k(0), jitter included, off the diagonal too),
    as in the reference; the values come out NaN and the status block says so, where the oracle's factorisation
    fails too."""
    from graphgp_b200 import graphgp_cuda as gc

    base = np.random.default_rng(4).standard_normal((300, 2)).astype(np.float32)
    pts = np.concatenate([base, base[:100], base[50:80]])
    n0, k = 16, 6
    bins, vals = rbf_table(scale=0.5)
    g = og.build_graph(pts, n0=n0, k=k)
    graph = gp.build_graph(torch.as_tensor(pts, device=cuda_device), n0=n0, k=k)
    assert graph.offsets == tuple(g.offsets)
    assert np.array_equal(graph.indices.cpu().numpy(), g.indices)
    assert np.array_equal(graph.neighbors.cpu().numpy(), g.neighbors)
    cov = (torch.as_tensor(bins, device=cuda_device), torch.as_tensor(vals, device=cuda_device))
    g64 = gp.Graph(graph.points.double(), graph.neighbors, graph.offsets, graph.indices)
    xi = np.random.default_rng(5).standard_normal(len(pts))
    v = gp.generate(g64, cov, torch.as_tensor(xi, device=cuda_device)).cpu().numpy()
    try:
        ref = orf.generate(g, (bins, vals), xi)
        oracle_fails = not np.all(np.isfinite(ref))
    except np.linalg.LinAlgError:
        oracle_fails = True
    assert oracle_fails
    assert np.isnan(v).any()
    assert gc.last_status()["nan_seen"] == 1


@pytest.mark.parametrize("n,n0,k", [(2, 1, 1), (3, 2, 2)])
def test_tiny_graphs(cuda_device, n, n0, k):
    pts = np.random.default_rng(n).standard_normal((n, 3)).astype(np.float32)
    _check(cuda_device, pts, n0=n0, k=k)
