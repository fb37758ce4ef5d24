"""Oracle: covariance lookup, dense root, refine / inverse / log-determinant and generate in float64.

Restates reference ``graphgp/refine.py``. Test infrastructure only; see ``oracle/__init__.py``.
All arithmetic is float64 (the reference tests run with ``jax_enable_x64``).
"""
from __future__ import annotations

import numpy as np

_CHUNK = 1 << 16


def cov_lookup(r, cov_bins, cov_vals):
    """``cov_lookup`` (refine.py:298-305) = ``jnp.interp(r, cov_bins, cov_vals)``, written out literally:
    bracket ``i = clip(searchsorted(xp, x, 'right'), 1, n-1)``, ``f = fp[i-1] + (x - xp[i-1]) / dx * df``,
    clamped to the end values outside ``[xp[0], xp[-1]]``."""
    xp = np.asarray(cov_bins, dtype=np.float64)
    fp = np.asarray(cov_vals, dtype=np.float64)
    x = np.asarray(r, dtype=np.float64)
    i = np.clip(np.searchsorted(xp, x, side="right"), 1, len(xp) - 1)
    df = fp[1:] - fp[:-1]
    dx = xp[1:] - xp[:-1]
    delta = x - xp[i - 1]
    eps = np.spacing(np.finfo(np.float64).eps)
    dx0 = np.abs(dx[i - 1]) <= eps
    f = np.where(dx0, fp[i - 1], fp[i - 1] + (delta / np.where(dx0, 1, dx[i - 1])) * df[i - 1])
    f = np.where(x < xp[0], fp[0], f)
    f = np.where(x > xp[-1], fp[-1], f)
    return f


def interp_weights(r, cov_bins):
    """Bracket index ``j`` and weight ``t`` such that ``cov_lookup(r) = (1 - t) vals[j] + t vals[j + 1]``
    (the derivative of ``jnp.interp`` with respect to ``fp``)."""
    xp = np.asarray(cov_bins, dtype=np.float64)
    x = np.asarray(r, dtype=np.float64)
    i = np.clip(np.searchsorted(xp, x, side="right"), 1, len(xp) - 1)
    dx = xp[i] - xp[i - 1]
    t = (x - xp[i - 1]) / dx
    t = np.where(x < xp[0], 0.0, t)
    t = np.where(x > xp[-1], 1.0, t)
    return i - 1, t


def pairwise_distances(a, b):
    """``jnp.linalg.norm(a[..., :, None, :] - b[..., None, :, :], axis=-1)`` (refine.py:289-290)."""
    diff = np.asarray(a, np.float64)[..., :, None, :] - np.asarray(b, np.float64)[..., None, :, :]
    return np.sqrt(np.sum(diff * diff, axis=-1))


def compute_cov_matrix(covariance, points_a, points_b):
    """``compute_cov_matrix`` (refine.py:288-295)."""
    cov_bins, cov_vals = covariance
    return cov_lookup(pairwise_distances(points_a, points_b), cov_bins, cov_vals)


# ------------------------------------------------------------------------------------------------
# dense root (refine.py:59-76, 186-195, 243-248)
# ------------------------------------------------------------------------------------------------
def generate_dense(points, covariance, xi):
    K = compute_cov_matrix(covariance, points, points)
    L = np.linalg.cholesky(K)
    return L @ np.asarray(xi, np.float64)


def generate_dense_inv(points, covariance, values):
    K = compute_cov_matrix(covariance, points, points)
    L = np.linalg.cholesky(K)
    return np.linalg.solve(L, np.asarray(values, np.float64))


def generate_dense_logdet(points, covariance):
    K = compute_cov_matrix(covariance, points, points)
    return np.linalg.slogdet(K)[1] / 2


# ------------------------------------------------------------------------------------------------
# per-point factorisation (refine.py:130-135, 221-227, 269-273)
# ------------------------------------------------------------------------------------------------
def factor_points(points, nbr_rows, self_idx, covariance):
    """mean_vec and std for points ``self_idx`` with neighbour id rows ``nbr_rows`` (see factor_rows)."""
    points = np.asarray(points, np.float64)
    nb = np.asarray(nbr_rows)
    k = nb.shape[1]
    joint = np.concatenate([points[nb], points[np.asarray(self_idx)][:, None, :]], axis=1)
    K = compute_cov_matrix(covariance, joint, joint)
    L = np.linalg.cholesky(K)
    mean_vec = np.linalg.solve(np.transpose(L[:, :k, :k], (0, 2, 1)), L[:, k, :k][..., None])[..., 0]
    return mean_vec, L[:, k, k]


def factor_rows(points, neighbors, covariance, n0, rows):
    """For refined rows ``rows`` (0-based into ``neighbors``): joint = [nbr_0..nbr_{k-1}, self];
    K = cov(joint, joint); L = chol(K); mean_vec = solve(L11^T, l21); std = L[k, k]."""
    points = np.asarray(points, np.float64)
    nb = np.asarray(neighbors)[rows]
    k = nb.shape[1]
    joint = np.concatenate([points[nb], points[n0 + np.asarray(rows)][:, None, :]], axis=1)
    K = compute_cov_matrix(covariance, joint, joint)
    with np.errstate(invalid="ignore"):
        L = np.linalg.cholesky(K) if len(K) else K
    if np.any(np.isnan(K)):
        pass
    mean_vec = np.linalg.solve(np.transpose(L[:, :k, :k], (0, 2, 1)), L[:, k, :k][..., None])[..., 0]
    std = L[:, k, k]
    return mean_vec, std


def _safe_factor(points, neighbors, covariance, n0, rows):
    """``factor_rows`` that maps a failed (non-SPD) factorisation to NaN like LAPACK-in-JAX does."""
    try:
        return factor_rows(points, neighbors, covariance, n0, rows)
    except np.linalg.LinAlgError:
        mv = np.empty((len(rows), np.asarray(neighbors).shape[1]))
        sd = np.empty(len(rows))
        for j, r in enumerate(rows):
            try:
                a, b = factor_rows(points, neighbors, covariance, n0, np.array([r]))
                mv[j], sd[j] = a[0], b[0]
            except np.linalg.LinAlgError:
                mv[j], sd[j] = np.nan, np.nan
        return mv, sd


def factor_all(points, neighbors, covariance, n0):
    m = len(neighbors)
    k = np.asarray(neighbors).shape[1]
    mean_vec = np.empty((m, k))
    std = np.empty(m)
    for s in range(0, m, _CHUNK):
        rows = np.arange(s, min(m, s + _CHUNK))
        mean_vec[rows], std[rows] = _safe_factor(points, neighbors, covariance, n0, rows)
    return mean_vec, std


# ------------------------------------------------------------------------------------------------
# refine / inverse / logdet (refine.py:79-159, 198-231, 251-275)
# ------------------------------------------------------------------------------------------------
def refine(points, neighbors, offsets, covariance, initial_values, xi, *, mode="fast_jit"):
    """``refine``: batch after batch, ``v_i = sum_m mean_vec_m v[nbr_m] + std_i xi_i``.

    ``mode="fast_jit"`` mirrors refine.py:123-145 (precomputed ``mean_vec``); ``mode="simple"`` mirrors
    refine.py:147-157 (``L[k, :k] @ solve(L[:k, :k], coarse_values)`` per batch)."""
    points = np.asarray(points, np.float64)
    neighbors = np.asarray(neighbors)
    n0 = len(points) - len(neighbors)
    if len(initial_values) != n0:
        raise ValueError("Length of initial_values must match number of initial points.")
    if len(xi) != len(points) - n0:
        raise ValueError("Length of xi must match number of refined points.")
    xi = np.asarray(xi, np.float64)
    values = np.zeros(len(points))
    values[:n0] = initial_values
    if mode == "fast_jit":
        mean_vec, std = factor_all(points, neighbors, covariance, n0)
        for b in range(1, len(offsets)):
            s, e = offsets[b - 1], offsets[b]
            rows = np.arange(s - n0, e - n0)
            values[s:e] = np.sum(mean_vec[rows] * values[neighbors[rows]], axis=1) + std[rows] * xi[rows]
    elif mode == "simple":
        k = neighbors.shape[1]
        for b in range(1, len(offsets)):
            s, e = offsets[b - 1], offsets[b]
            rows = np.arange(s - n0, e - n0)
            nb = neighbors[rows]
            joint = np.concatenate([points[nb], points[s:e][:, None, :]], axis=1)
            K = compute_cov_matrix(covariance, joint, joint)
            L = np.linalg.cholesky(K)
            z = np.linalg.solve(L[:, :k, :k], values[nb][..., None])[..., 0]
            mean = np.sum(L[:, k, :k] * z, axis=1)
            values[s:e] = mean + L[:, k, k] * xi[rows]
    else:
        raise ValueError(mode)
    return values


def refine_inv(points, neighbors, offsets, covariance, values):
    """``refine_inv`` (refine.py:198-231): xi_i = (v_i - sum_m mean_vec_m v[nbr_m]) / std_i."""
    points = np.asarray(points, np.float64)
    values = np.asarray(values, np.float64)
    n0 = len(points) - len(neighbors)
    if len(values) != len(points):
        raise ValueError("Length of values must match number of points.")
    mean_vec, std = factor_all(points, neighbors, covariance, n0)
    mean = np.sum(mean_vec * values[np.asarray(neighbors)], axis=1)
    return values[:n0].copy(), (values[n0:] - mean) / std


def refine_logdet(points, neighbors, offsets, covariance):
    """``refine_logdet`` (refine.py:251-275): sum of log std."""
    n0 = len(points) - len(neighbors)
    _, std = factor_all(points, neighbors, covariance, n0)
    return float(np.sum(np.log(std)))


# ------------------------------------------------------------------------------------------------
# generate (refine.py:21-56, 162-183, 234-240)
# ------------------------------------------------------------------------------------------------
def generate(graph, covariance, xi, *, mode="fast_jit"):
    xi = np.asarray(xi, np.float64)
    if len(xi) != len(graph.points):
        raise ValueError("Length of xi must match number of points in graph.")
    n0 = len(graph.points) - len(graph.neighbors)
    if graph.indices is not None:
        xi = xi[graph.indices]
    initial_values = generate_dense(graph.points[:n0], covariance, xi[:n0])
    values = refine(graph.points, graph.neighbors, graph.offsets, covariance, initial_values, xi[n0:], mode=mode)
    if graph.indices is not None:
        out = np.empty_like(values)
        out[graph.indices] = values
        values = out
    if np.any(np.isnan(values)):
        values = np.full_like(values, np.nan)
    return values


def generate_inv(graph, covariance, values):
    values = np.asarray(values, np.float64)
    if len(values) != len(graph.points):
        raise ValueError("Length of values must match number of points in graph.")
    n0 = len(graph.points) - len(graph.neighbors)
    if graph.indices is not None:
        values = values[graph.indices]
    initial_values, xi = refine_inv(graph.points, graph.neighbors, graph.offsets, covariance, values)
    initial_xi = generate_dense_inv(graph.points[:n0], covariance, initial_values)
    xi = np.concatenate([initial_xi, xi])
    if graph.indices is not None:
        out = np.empty_like(xi)
        out[graph.indices] = xi
        xi = out
    if np.any(np.isnan(xi)):
        xi = np.full_like(xi, np.nan)
    return xi


def generate_logdet(graph, covariance):
    n0 = len(graph.points) - len(graph.neighbors)
    dense = generate_dense_logdet(graph.points[:n0], covariance)
    return float(dense + refine_logdet(graph.points, graph.neighbors, graph.offsets, covariance))
