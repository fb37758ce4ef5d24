"""Host-side parts of the reference-shaped API (no GPU): check_graph, compute_cov_matrix, graph files, and the
refusal of cuda=False."""
import numpy as np
import pytest
import torch

import graphgp_b200 as gp
from oracle import refine as orf

from helpers import oracle_graph, rbf_table


def _graph(n=2000, d=2, n0=64, k=8):
    _, g = oracle_graph(n, d, n0, k)
    return gp.Graph(torch.as_tensor(g.points), torch.as_tensor(g.neighbors), tuple(g.offsets),
                    torch.as_tensor(g.indices))


def test_check_graph_accepts_and_rejects():
    g = _graph()
    gp.check_graph(g)
    bad = gp.Graph(g.points, g.neighbors.clone(), g.offsets, g.indices)
    bad.neighbors[5, 0] = g.offsets[0] + 5  # a point depending on itself
    with pytest.raises(AssertionError):
        gp.check_graph(bad)
    with pytest.raises(AssertionError):
        gp.check_graph(gp.Graph(g.points, g.neighbors, (g.offsets[0] + 1,) + g.offsets[1:], g.indices))


def test_compute_cov_matrix_matches_oracle():
    rng = np.random.default_rng(4)
    a, b = rng.standard_normal((50, 3)), rng.standard_normal((40, 3)) * 3.0
    bins, vals = rbf_table(scale=0.7)
    out = gp.compute_cov_matrix((torch.as_tensor(bins), torch.as_tensor(vals)), torch.as_tensor(a),
                                torch.as_tensor(b))
    ref = orf.compute_cov_matrix((bins, vals), a, b)
    assert np.allclose(out.numpy(), ref, rtol=1e-12, atol=1e-14)


def test_graph_file_round_trip(tmp_path):
    g = _graph()
    gp.save_graph(tmp_path / "g.npz", g)
    h = gp.load_graph(tmp_path / "g.npz", device="cpu")
    assert h.offsets == g.offsets
    assert torch.equal(h.points, g.points) and torch.equal(h.neighbors, g.neighbors)
    assert torch.equal(h.indices, g.indices)


def test_cpu_path_refused():
    with pytest.raises(NotImplementedError):
        gp.build_graph(torch.zeros(10, 2), n0=4, k=2, cuda=False)
