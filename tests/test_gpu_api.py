"""The reference-shaped API on the GPU: build_graph gives a Graph that check_graph accepts and that equals the
oracle's; generate / generate_inv / generate_logdet and the dense functions match the FP64 oracle; a graph
saved to a file and loaded back gives identical results."""
import numpy as np
import pytest
import torch

import graphgp_b200 as gp
from oracle import refine as orf

from conftest import rel_err
from helpers import oracle_graph, matern32_table

pytestmark = pytest.mark.gpu


def test_api_end_to_end(cuda_device, tmp_path):
    n, d, n0, k = 3000, 3, 128, 16
    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = matern32_table(cutoff=0.4)
    cov = (torch.as_tensor(bins, device=cuda_device), torch.as_tensor(vals, device=cuda_device))
    graph = gp.build_graph(torch.as_tensor(pts, device=cuda_device), n0=n0, k=k)
    gp.check_graph(graph)
    assert graph.offsets == tuple(g.offsets)
    assert np.array_equal(graph.neighbors.cpu().numpy(), g.neighbors)
    assert np.array_equal(graph.indices.cpu().numpy(), g.indices)
    # FP64 graph points for FP64 parity of the operations
    g64 = gp.Graph(graph.points.double(), graph.neighbors, graph.offsets, graph.indices)
    xi = np.random.default_rng(3).standard_normal(n)
    v = gp.generate(g64, cov, torch.as_tensor(xi, device=cuda_device))
    ref = orf.generate(g, (bins, vals), xi)
    assert rel_err(v.cpu().numpy(), ref) < 1e-9
    x2 = gp.generate_inv(g64, cov, v)
    assert rel_err(x2.cpu().numpy(), xi) < 1e-9
    ld = float(gp.generate_logdet(g64, cov))
    assert abs(ld - orf.generate_logdet(g, (bins, vals))) <= 1e-9 * abs(ld)
    p0 = g64.points[:n0]
    assert rel_err(gp.generate_dense(p0, cov, torch.as_tensor(xi[:n0], device=cuda_device)).cpu().numpy(),
                   orf.generate_dense(g.points[:n0].astype(np.float64), (bins, vals), xi[:n0])) < 1e-11
    gp.save_graph(tmp_path / "g.npz", g64)
    h = gp.load_graph(tmp_path / "g.npz", device=cuda_device)
    assert torch.equal(gp.generate(h, cov, torch.as_tensor(xi, device=cuda_device)), v)
