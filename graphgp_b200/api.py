"""The reference's public API (graphgp/__init__.py) on CUDA ``torch.Tensor`` s, running this package's kernels.

Same names, argument meaning, results and errors as the reference's ``cuda=True`` path: ``Graph``,
``check_graph``, ``build_graph``, ``build_tree``, ``query_preceding_neighbors``, ``query_neighbors``,
``compute_depths``, ``order_by_depth``, ``generate`` / ``generate_inv`` / ``generate_logdet``,
``generate_dense`` / ``_inv`` / ``_logdet``, ``refine`` / ``refine_inv`` / ``refine_logdet`` and
``compute_cov_matrix`` (reference graph.py:20-137, tree.py:19-76, refine.py:21-305). A covariance is the pair
``(cov_bins, cov_vals)``. There is no CPU path: ``cuda=False`` raises.

Beyond the reference: ``generate_vjp`` (the adjoint, which also backs autograd through ``generate``,
``generate_logdet`` and ``generate_and_logdet``), and ``save_graph`` / ``load_graph`` to keep a built graph across
processes as an ``.npz`` file.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import torch

from . import autograd as _ag
from . import graphgp_cuda as _gc


def _need_cuda(cuda):
    if not cuda:
        raise NotImplementedError("graphgp_b200 runs the cuda=True path only; it has no CPU implementation")


@dataclass
class Graph:
    """Nearest-neighbour dependency graph (reference graph.py:20-41): ``points`` (N, d) in graph order,
    ``neighbors`` (N - offsets[0], k), ``offsets`` (tuple, end index of each batch), ``indices`` (N,) original
    point ids or None."""

    points: torch.Tensor
    neighbors: torch.Tensor
    offsets: Tuple[int, ...]
    indices: Optional[torch.Tensor] = None


def check_graph(graph: Graph):
    """Verify the graph can be used (reference graph.py:44-70): neighbours start at the first offset, offsets are
    non-decreasing and within N, points are in topological order and no neighbour is in its own batch."""
    points, neighbors = graph.points, graph.neighbors
    offsets = torch.as_tensor(graph.offsets, dtype=torch.int64, device=neighbors.device)
    assert int(offsets[0]) == len(points) - len(neighbors), "Neighbors should start from first offset"
    assert bool(torch.all(offsets[1:] >= offsets[:-1])), "Offsets must be non-decreasing"
    assert int(offsets[-1]) <= len(points), "Last offset must be less than or equal to the number of points"
    max_neighbors = neighbors.long().max(dim=1).values
    index = torch.arange(len(neighbors), device=neighbors.device) + offsets[0]
    assert bool(torch.all(max_neighbors < index)), "Points are not in topological order"
    batch = torch.searchsorted(offsets, index, right=True) - 1
    assert bool(torch.all(max_neighbors < offsets[batch])), "Neighbors must not be in the same batch"


def build_graph(points: torch.Tensor, *, n0: int, k: int, cuda: bool = True) -> Graph:
    """k-d tree, preceding k-NN, depths, ordering and offsets in one device call (reference graph.py:73-98)."""
    _need_cuda(cuda)
    p, idx, nbrs, _, offs = _gc.build_graph(points, n0=n0, k=k, return_offsets=True)
    return Graph(p, nbrs, offs, idx)


def build_tree(points, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.build_tree(points)


def query_preceding_neighbors(points, split_dims, *, n0: int, k: int, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.query_preceding_neighbors(points, split_dims, n0=n0, k=k)


def query_neighbors(points, split_dims, query_indices, max_indices, *, k: int, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.query_neighbors(points, split_dims, query_indices, max_indices, k=k)


def compute_depths(neighbors, *, n0: int, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.compute_depths_parallel(neighbors, n0=n0)


def order_by_depth(points, indices, neighbors, depths, *, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.order_by_depth(points, indices, neighbors, depths)


def _wants_grad(*ts):
    return torch.is_grad_enabled() and any(isinstance(t, torch.Tensor) and t.requires_grad for t in ts)


def generate(graph: Graph, covariance, xi, *, cuda: bool = True, fast_jit: bool = True):
    """Values (N,) in the original point order (reference refine.py:21-56). ``fast_jit`` has one meaning here:
    both of the reference's forms compute the same values. Differentiable: when ``xi`` or the table values
    require grad, the call is recorded for autograd and its backward runs the adjoint kernels
    (``graphgp_b200.autograd.GenerateFn``)."""
    _need_cuda(cuda)
    if _wants_grad(xi, covariance[1]):
        return _ag.generate(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                            covariance[1], xi)
    return _gc.generate(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0], covariance[1],
                        xi)


def generate_inv(graph: Graph, covariance, values, *, cuda: bool = True):
    """xi (N,) from values (N,), original order (reference refine.py:162-183)."""
    _need_cuda(cuda)
    return _gc.generate_inv(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                            covariance[1], values)


def generate_logdet(graph: Graph, covariance, *, cuda: bool = True):
    """Log-determinant of the generate map, FP64 (reference refine.py:234-240). Differentiable in the table
    values (``graphgp_b200.autograd.GenerateLogdetFn``)."""
    _need_cuda(cuda)
    if _wants_grad(covariance[1]):
        return _ag.generate_logdet(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                                   covariance[1])
    return _gc.generate_logdet(graph.points, graph.neighbors, graph.offsets, covariance[0], covariance[1])


def generate_and_logdet(graph: Graph, covariance, xi, *, cuda: bool = True):
    """``(generate(graph, covariance, xi), generate_logdet(graph, covariance))`` in one call (one forward pass in
    FP32); under autograd the backward pass runs a single adjoint sweep for both outputs (a likelihood
    0.5|v - y|^2 + logdet)."""
    _need_cuda(cuda)
    if _wants_grad(xi, covariance[1]):
        return _ag.generate_and_logdet(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                                       covariance[1], xi)
    return _gc.generate_and_logdet(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                                   covariance[1], xi)


def generate_vjp(graph: Graph, covariance, xi, g_values, g_logdet: float = 0.0, *, values=None):
    """Gradients of <g_values, generate(xi)> + g_logdet * generate_logdet with respect to xi and the table values
    (the adjoint the reference obtains from JAX autodiff). ``values``: generate's output, if at hand."""
    return _gc.generate_vjp(graph.points, graph.indices, graph.neighbors, graph.offsets, covariance[0],
                            covariance[1], xi, g_values, g_logdet, values=values)


def generate_dense(points, covariance, xi):
    """L @ xi with L the FP64 Cholesky factor of the dense covariance (reference refine.py:59-76)."""
    return _gc.dense("generate", points, covariance[0], covariance[1], xi)


def generate_dense_inv(points, covariance, values):
    """L^-1 values (reference refine.py:186-195)."""
    return _gc.dense("inverse", points, covariance[0], covariance[1], values)


def generate_dense_logdet(points, covariance):
    """sum log L_ii = slogdet(K) / 2 (reference refine.py:243-248)."""
    return _gc.dense("logdet", points, covariance[0], covariance[1])


def refine(points, neighbors, offsets, covariance, initial_values, xi, *, cuda: bool = True, fast_jit: bool = True):
    _need_cuda(cuda)
    return _gc.refine(points, neighbors, offsets, covariance[0], covariance[1], initial_values, xi)


def refine_inv(points, neighbors, offsets, covariance, values, *, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.refine_inv(points, neighbors, offsets, covariance[0], covariance[1], values)


def refine_logdet(points, neighbors, offsets, covariance, *, cuda: bool = True):
    _need_cuda(cuda)
    return _gc.refine_logdet(points, neighbors, offsets, covariance[0], covariance[1])


def compute_cov_matrix(covariance, points_a, points_b):
    """Covariance matrix between two point sets by linear interpolation of the table at the pairwise distances,
    with end values held outside it (reference refine.py:288-305). A convenience for small sets (it materialises
    the matrix); the refinement kernels never form it."""
    bins, vals = covariance
    r = torch.cdist(points_a.double().unsqueeze(0), points_b.double().unsqueeze(0)).squeeze(0)
    bins = bins.to(r.device, torch.float64)
    vals = vals.to(r.device, torch.float64)
    j = torch.clamp(torch.searchsorted(bins, r, right=True) - 1, 0, len(bins) - 2)
    b0, b1 = bins[j], bins[j + 1]
    v0, v1 = vals[j], vals[j + 1]
    t = torch.where(b1 > b0, (r - b0) / (b1 - b0), torch.zeros_like(r))
    out = v0 + t * (v1 - v0)
    out = torch.where(r <= bins[0], vals[0], out)
    out = torch.where(r >= bins[-1], vals[-1], out)
    return out.to(points_a.dtype)


def save_graph(path, graph: Graph):
    """Write a graph to ``path`` (``.npz``): points, neighbors, offsets and indices."""
    arrays = {"points": graph.points.cpu().numpy(), "neighbors": graph.neighbors.cpu().numpy(),
              "offsets": np.asarray(graph.offsets, np.int64)}
    if graph.indices is not None:
        arrays["indices"] = graph.indices.cpu().numpy()
    np.savez(path, **arrays)


def load_graph(path, device=None) -> Graph:
    """Read a graph written by ``save_graph`` onto ``device`` (default: the current CUDA device)."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    with np.load(path) as f:
        idx = torch.as_tensor(f["indices"], device=device) if "indices" in f.files else None
        return Graph(torch.as_tensor(f["points"], device=device), torch.as_tensor(f["neighbors"], device=device),
                     tuple(int(x) for x in f["offsets"]), idx)
