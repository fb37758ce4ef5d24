"""Autograd through generate and generate_logdet (graphgp_b200.autograd): the backward passes run the adjoint
kernels. The reference differentiates generate with JAX autodiff (graphgp/refine.py:21-56; its test takes
jax.jacfwd of generate, tests/test_refine.py:77); here torch.autograd.gradcheck compares the adjoint with central
differences of the FP64 forward, and the FP32 loss.backward() must give what the adjoint call gives.
"""
import numpy as np
import pytest

from helpers import oracle_graph, rbf_table

pytestmark = pytest.mark.gpu


def _graph(dev, dtype, n=300, d=2, n0=40, k=8):
    import torch

    import graphgp_b200 as gg

    pts, g = oracle_graph(n, d, n0, k, seed=7)
    graph = gg.Graph(torch.as_tensor(g.points, device=dev, dtype=dtype), torch.as_tensor(g.neighbors, device=dev),
                     g.offsets, torch.as_tensor(g.indices, device=dev))
    # a 1,001-entry table: linear interpolation of a coarser RBF table is not positive definite at this jitter
    bins, vals = rbf_table(scale=0.3, n_bins=1001, jitter=1e-3)
    return graph, torch.as_tensor(bins, device=dev, dtype=dtype), torch.as_tensor(vals, device=dev, dtype=dtype)


def test_gradcheck_generate_fp64(cuda_device):
    import torch

    import graphgp_b200 as gg

    graph, B, V = _graph(cuda_device, torch.float64)
    xi = torch.randn(len(graph.points), dtype=torch.float64, device=cuda_device, requires_grad=True)
    vals = V.clone().requires_grad_(True)
    # torch's default tolerances (atol 1e-5, rtol 1e-3): with Schur complements near the jitter the loss is far from
    # linear in the table, and central differences with step 1e-6 carry ~1e-5 relative truncation error on a few
    # entries. The adjoint's per-block FP64 sums are taken in a scheduling-dependent order: allow rounding-level
    # differences between repeated backward passes.
    assert torch.autograd.gradcheck(lambda x, v: gg.generate(graph, (B, v), x), (xi, vals), eps=1e-6,
                                    nondet_tol=1e-10)


def test_gradcheck_generate_logdet_fp64(cuda_device):
    import torch

    import graphgp_b200 as gg

    graph, B, V = _graph(cuda_device, torch.float64)
    vals = V.clone().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda v: gg.generate_logdet(graph, (B, v)), (vals,), eps=1e-6, nondet_tol=1e-10)


def test_backward_equals_adjoint_fp32(cuda_device):
    """loss = 0.5 |generate(xi) - y|^2 + logdet through generate_and_logdet: loss.backward() equals one
    generate_vjp call with both cotangents (the same kernels on the same inputs)."""
    import torch

    import graphgp_b200 as gg
    from graphgp_b200 import graphgp_cuda as gc

    graph, B, V = _graph(cuda_device, torch.float32, n=3000, d=2, n0=128, k=16)
    n = len(graph.points)
    gen = torch.Generator(device=cuda_device).manual_seed(3)
    y = torch.randn(n, generator=gen, device=cuda_device)
    xi = torch.randn(n, generator=gen, device=cuda_device).requires_grad_(True)
    vals = V.clone().requires_grad_(True)
    v, ld = gg.generate_and_logdet(graph, (B, vals), xi)
    assert bool(torch.isfinite(v).all()) and bool(torch.isfinite(ld))
    loss = 0.5 * torch.sum((v - y) ** 2) + ld
    loss.backward()
    with torch.no_grad():
        v0 = gc.generate(graph.points, graph.indices, graph.neighbors, graph.offsets, B, V, xi.detach())
        gx, gv = gc.generate_vjp(graph.points, graph.indices, graph.neighbors, graph.offsets, B, V, xi.detach(),
                                 v0 - y, 1.0, values=v0)
    assert torch.equal(v.detach(), v0)
    # the adjoint scatters cotangents with atomics in a scheduling-dependent order: FP32 rounding differences
    np.testing.assert_allclose(xi.grad.cpu().numpy(), gx.cpu().numpy(), rtol=1e-5, atol=1e-5 * float(gx.abs().max()))
    np.testing.assert_allclose(vals.grad.double().cpu().numpy(), gv.float().double().cpu().numpy(), rtol=1e-5,
                               atol=1e-5 * float(gv.abs().max()))


@pytest.mark.parametrize("k,d", [(16, 2), (20, 3), (13, 3), (7, 2)])
def test_backward_with_and_without_residuals(cuda_device, k, d):
    """GenerateAndLogdetFn's backward reading the forward's residuals equals the refactorising backward (FP32
    rounding: a = K11^-1 v_N is solved in another order)."""
    import torch

    import graphgp_b200 as gg
    from graphgp_b200 import autograd as ag

    graph, B, V = _graph(cuda_device, torch.float32, n=4000, d=d, n0=100, k=k)
    n = len(graph.points)
    gen = torch.Generator(device=cuda_device).manual_seed(k)
    y = torch.randn(n, generator=gen, device=cuda_device)
    xi0 = torch.randn(n, generator=gen, device=cuda_device)
    grads = []
    saved = ag.RESIDUALS
    try:
        for flag in (True, False):
            ag.RESIDUALS = flag
            xi = xi0.clone().requires_grad_(True)
            vals = V.clone().requires_grad_(True)
            v, ld = gg.generate_and_logdet(graph, (B, vals), xi)
            (0.5 * torch.sum((v - y) ** 2) + ld).backward()
            grads.append((xi.grad.cpu().numpy(), vals.grad.double().cpu().numpy()))
    finally:
        ag.RESIDUALS = saved
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-5 * float(np.abs(b).max()))
