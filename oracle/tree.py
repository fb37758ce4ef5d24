"""Oracle: k-d tree build and preceding k-NN query (restates reference ``graphgp/tree.py``).

Test infrastructure only; see ``oracle/__init__.py``.

Conventions that make the restatement exact:
* arithmetic is done in the dtype of ``points`` (float32 in production, float64 in the reference tests);
* a squared distance is summed left to right over dimensions, each term an unfused ``diff * diff``;
* node levels use exact integer arithmetic (``bit_length``), which equals the reference's
  ``jnp.frexp(current + 1)[1] - 1`` (``tree.py:188``) whenever ``current + 1`` is exactly representable in
  the float type JAX promotes to (always in float64; up to 2**24 in float32).
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------------------------
# implicit-tree index arithmetic -- reference tree.py:187-208
# ---------------------------------------------------------------------------------------------
def _level(current):
    current = np.asarray(current, dtype=np.int64)
    # floor(log2(current + 1)); bit_length of (current + 1) minus one
    c1 = current + 1
    lvl = np.zeros_like(c1)
    pos = c1 > 0
    lvl[pos] = np.floor(np.log2(c1[pos].astype(np.float64))).astype(np.int64)
    # guard against log2 rounding for large values
    lvl[pos] -= (np.left_shift(1, lvl[pos]) > c1[pos]).astype(np.int64)
    lvl[pos] += (np.left_shift(1, lvl[pos] + 1) <= c1[pos]).astype(np.int64)
    lvl[~pos] = -1
    return lvl


def compute_left(current):
    """``_compute_left`` (tree.py:187-191): current + 2**level."""
    current = np.asarray(current, dtype=np.int64)
    return current + np.left_shift(1, _level(current))


def compute_right(current):
    """``_compute_right`` (tree.py:194-198): current + 2 * 2**level."""
    current = np.asarray(current, dtype=np.int64)
    return current + 2 * np.left_shift(1, _level(current))


def compute_parent(current):
    """``_compute_parent`` (tree.py:201-208); the root's parent is -1."""
    current = np.asarray(current, dtype=np.int64)
    lvl = _level(current)
    lvl_safe = np.maximum(lvl, 1)
    n_above = np.left_shift(1, lvl_safe) - 1
    n_parent_level = np.left_shift(1, lvl_safe - 1)
    parent = np.where(current < n_above + n_parent_level, current - n_parent_level, current - 2 * n_parent_level)
    return np.where(current == 0, -1, parent)


# ---------------------------------------------------------------------------------------------
# tree build -- reference tree.py:153-184 and _update_nodes tree.py:211-234
# ---------------------------------------------------------------------------------------------
def update_nodes(nodes, index, level, n_points):
    """``_update_nodes`` (tree.py:211-234)."""
    n_above = (1 << level) - 1
    n_level = 1 << level
    n_remaining = n_points - n_above
    q = n_remaining // n_level
    r = n_remaining % n_level
    i = nodes - n_above
    midpoint = np.where(i < r, i * (q + 1) + (q + 1) // 2, r * (q + 1) + (i - r) * q + q // 2) + n_above
    return np.where(
        (index < n_above) | (index == midpoint),
        nodes,
        np.where(index < midpoint, nodes + n_level, nodes + 2 * n_level),
    )


def build_tree(points):
    """``build_tree`` / ``_build_tree`` (tree.py:18-38, 153-184).

    Returns ``(points_tree, split_dims, indices)``; ``split_dims`` and ``indices`` are int64 here.
    """
    points = np.asarray(points)
    if points.ndim != 2:
        raise ValueError(f"Points must have shape (N, d). Got shape {points.shape}.")
    n_points, n_dim = points.shape
    n_levels = int(n_points).bit_length()
    array_index = np.arange(n_points, dtype=np.int64)
    nodes = np.zeros(n_points, dtype=np.int64)
    indices = np.arange(n_points, dtype=np.int64)
    split_dims = -np.ones(n_points, dtype=np.int64)
    pts = points.copy()
    for level in range(n_levels):
        # segment_max / segment_min over node ids (tree.py:162-163); empty segments give -inf / +inf
        dim_max = np.full((n_points, n_dim), -np.inf, dtype=pts.dtype)
        dim_min = np.full((n_points, n_dim), np.inf, dtype=pts.dtype)
        np.maximum.at(dim_max, nodes, pts)
        np.minimum.at(dim_min, nodes, pts)
        new_split_dims = np.argmax(dim_max - dim_min, axis=-1)  # first maximum (tree.py:164)
        split_dims = np.where(array_index < (1 << level) - 1, split_dims, new_split_dims)
        along = pts[array_index, split_dims[nodes]]
        # stable sort by (node, coordinate, current position) (tree.py:172); np.lexsort: last key primary
        perm = np.lexsort((array_index, along, nodes))
        nodes = nodes[perm]
        indices = indices[perm]
        pts = pts[perm]
        nodes = update_nodes(nodes, array_index, level, n_points)
    return pts, split_dims, indices


# ---------------------------------------------------------------------------------------------
# k-NN query -- reference tree.py:41-150, evaluated for all queries in lock step (like jax.vmap)
# ---------------------------------------------------------------------------------------------
def _sqdist(points, a, b):
    """Squared distance in points' dtype, summed left to right, unfused (tree.py:83)."""
    diff = points[a] - points[b]
    acc = diff[:, 0] * diff[:, 0]
    for j in range(1, points.shape[1]):
        acc = acc + diff[:, j] * diff[:, j]
    return acc


def query_neighbors(points, split_dims, query_indices, max_indices, *, k):
    """``query_neighbors`` (tree.py:66-76) -> ``_single_query_neighbors`` (79-105) for every query.

    Returns int64 ``(Q, k)`` neighbour ids sorted by (distance, index).
    """
    points = np.asarray(points)
    split_dims = np.asarray(split_dims, dtype=np.int64)
    q_idx = np.asarray(query_indices, dtype=np.int64)
    m_idx = np.asarray(max_indices, dtype=np.int64)
    Q = len(q_idx)
    dtype = points.dtype
    nbrs = -np.ones((Q, k), dtype=np.int64)
    sqd = np.full((Q, k), np.inf, dtype=dtype)
    radius = np.full(Q, np.inf, dtype=dtype)
    current = np.zeros(Q, dtype=np.int64)
    previous = -np.ones(Q, dtype=np.int64)
    active = np.nonzero(current != -1)[0]
    while len(active):
        c = current[active]
        p = previous[active]
        q = q_idx[active]
        mx = m_idx[active]
        parent = compute_parent(c)
        # update_func (tree.py:81-95) when arriving from the parent (tree.py:121-123)
        upd = p == parent
        if upd.any():
            ua = active[upd]
            uc = c[upd]
            d2 = _sqdist(points, q[upd], uc)
            slots = sqd[ua]
            amax = np.argmax(slots, axis=1)  # first maximum
            cur = slots[np.arange(len(ua)), amax]
            rep = d2 < cur
            ra, rs = ua[rep], amax[rep]
            nbrs[ra, rs] = uc[rep]
            sqd[ra, rs] = d2[rep]
            radius[ua] = sqd[ua].max(axis=1)
        sd = split_dims[c]
        split_distance = points[q, sd] - points[c, sd]
        left = compute_left(c)
        right = compute_right(c)
        near = np.where(split_distance < 0, left, right)
        far = np.where(split_distance < 0, right, left)
        far_in_range = split_distance * split_distance <= radius[active]
        nxt = np.where(
            (p == near) | ((p == parent) & (near >= mx)),
            np.where((far < mx) & far_in_range, far, parent),
            np.where(p == parent, near, parent),
        )
        previous[active] = c
        current[active] = nxt
        active = active[nxt != -1]
    # final ordering by (distance, index) (tree.py:103-104)
    diff = points[nbrs] - points[q_idx][:, None, :]
    acc = diff[..., 0] * diff[..., 0]
    for j in range(1, points.shape[1]):
        acc = acc + diff[..., j] * diff[..., j]
    dist = np.sqrt(acc)
    order = np.lexsort((nbrs, dist), axis=-1)
    return np.take_along_axis(nbrs, order, axis=-1)


def query_preceding_neighbors(points, split_dims, *, n0, k):
    """``query_preceding_neighbors`` (tree.py:41-63)."""
    if n0 < k:
        raise ValueError(f"n0 must be at least k. Got n0={n0}, k={k}.")
    q = np.arange(n0, len(points), dtype=np.int64)
    return query_neighbors(points, split_dims, q, q, k=k)
