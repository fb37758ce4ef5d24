"""Oracle: depths, ordering by depth, offsets and graph validation (restates reference ``graphgp/graph.py``).

Test infrastructure only; see ``oracle/__init__.py``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import tree as _tree


@dataclass
class Graph:
    """``Graph`` (graph.py:20-41): points in graph order, neighbours (N - offsets[0], k), offsets, indices."""

    points: np.ndarray
    neighbors: np.ndarray
    offsets: Tuple[int, ...]
    indices: Optional[np.ndarray] = None


def check_graph(graph: Graph):
    """``check_graph`` (graph.py:44-70)."""
    points, neighbors = graph.points, graph.neighbors
    offsets = np.asarray(graph.offsets)
    assert offsets[0] == len(points) - len(neighbors), "Neighbors should start from first offset"
    assert np.all(offsets[1:] >= offsets[:-1]), "Offsets must be non-decreasing"
    assert offsets[-1] <= len(points), "Last offset must be less than or equal to the number of points"
    max_neighbors = np.max(neighbors, axis=1)
    index = np.arange(len(neighbors)) + offsets[0]
    assert np.all(max_neighbors < index), "Points are not in topological order"
    offsets_index = np.searchsorted(offsets, index, side="right") - 1
    assert np.all(max_neighbors < offsets[offsets_index]), "Neighbors must not be in the same batch"


def compute_depths(neighbors, *, n0, max_iter=None):
    """``compute_depths`` (graph.py:101-120): Jacobi fixed point of depth[i] = 1 + max(depth[nbrs[i]])."""
    neighbors = np.asarray(neighbors, dtype=np.int64)
    n = n0 + len(neighbors)
    depths = np.zeros(n, dtype=np.int32)
    old = depths - 1
    it = 0
    while np.any(old != depths):
        new = depths.copy()
        if len(neighbors):
            new[n0:] = 1 + np.max(depths[neighbors], axis=1)
        old, depths = depths, new
        it += 1
        if max_iter is not None and it > max_iter:
            raise RuntimeError("compute_depths did not converge")
    return depths


def order_by_depth(points, indices, neighbors, depths):
    """``order_by_depth`` (graph.py:123-137): stable argsort by depth, permute, remap neighbour ids."""
    n0 = len(points) - len(neighbors)
    order = np.argsort(depths, kind="stable")
    points, indices, depths = points[order], indices[order], depths[order]
    neighbors = neighbors[order[n0:] - n0]
    inv_order = np.arange(len(points), dtype=np.int64)
    inv_order[order] = np.arange(len(points), dtype=np.int64)
    neighbors = inv_order[neighbors]
    return points, indices, neighbors, depths


def compute_offsets(depths):
    """offsets[b] = searchsorted_left(depths, b + 1) for b = 0..max_depth (graph.py:95-96)."""
    depths = np.asarray(depths)
    offs = np.searchsorted(depths, np.arange(1, int(depths.max()) + 2))
    return tuple(int(x) for x in offs)


def build_graph(points, *, n0, k):
    """``build_graph`` (graph.py:73-98)."""
    pts, split_dims, indices = _tree.build_tree(points)
    neighbors = _tree.query_preceding_neighbors(pts, split_dims, n0=n0, k=k)
    depths = compute_depths(neighbors, n0=n0)
    pts, indices, neighbors, depths = order_by_depth(pts, indices, neighbors, depths)
    return Graph(pts, neighbors, compute_offsets(depths), indices)
