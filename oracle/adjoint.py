"""Oracle: reverse-mode gradient of generate (+ a log-determinant term), written out by hand in float64.

Test infrastructure only; see ``oracle/__init__.py``. This is the derivative JAX's autodiff takes through
reference ``graphgp/refine.py:21-76`` (dense root) and ``123-145`` (per-point conditioning, batch scan) with
respect to ``xi`` and the table values ``cov_vals`` (``jnp.interp`` is linear in ``fp``), for the loss
``<g_values, generate(xi)> + g_logdet * generate_logdet``.

Per refined point i with neighbours N: w = K11^-1 k12, a = K11^-1 v_N, mean = w . v_N, sigma^2 = K22 - k12.w.
With mbar = vbar_i and sbar = vbar_i xi_i + g_logdet / sigma:
  d mean / d f(r_ab) = -(w_a a_b + w_b a_a)  (a != b neighbours),  -w_a a_a  (diagonal)
  d sigma / d f(r_ab) = w_a w_b / sigma,                            w_a^2 / (2 sigma)
  d mean / d f(r_a,self) = a_a,  d sigma / d f(r_a,self) = -w_a / sigma,  d sigma / d K22 = 1 / (2 sigma)
and vbar of each neighbour receives w_m vbar_i, xibar_i = sigma vbar_i. Root (v0 = L xi0):
  xibar0 = L^T vbar0,  Kbar0 = L^-T (tril(y xi0^T) - diag(y xi0)/2 + g_logdet/2 I) L^-1,  y = L^T vbar0.
"""
from __future__ import annotations

import numpy as np

from . import refine as orf


def _scatter_table(grad, r, coef, bins):
    j, t = orf.interp_weights(r.ravel(), bins)
    c = coef.ravel()
    np.add.at(grad, j, c * (1 - t))
    np.add.at(grad, np.minimum(j + 1, len(bins) - 1), c * t)


def generate_vjp(graph, covariance, xi, g_values, g_logdet=0.0):
    """Returns (grad_xi (N,), grad_vals (n_bins,)) in the original point order."""
    bins, vals = (np.asarray(c, np.float64) for c in covariance)
    pts = np.asarray(graph.points, np.float64)
    nbrs = np.asarray(graph.neighbors)
    offs = graph.offsets
    n = len(pts)
    n0 = n - len(nbrs)
    k = nbrs.shape[1]
    idx = np.arange(n) if graph.indices is None else np.asarray(graph.indices)
    xi_g = np.asarray(xi, np.float64)[idx]
    # forward values in graph order
    v0 = orf.generate_dense(pts[:n0], (bins, vals), xi_g[:n0])
    values = orf.refine(pts, nbrs, offs, (bins, vals), v0, xi_g[n0:])
    vbar = np.asarray(g_values, np.float64)[idx].copy()
    grad_xi_g = np.zeros(n)
    grad_vals = np.zeros(len(bins))
    for b in range(len(offs) - 1, 0, -1):
        s, e = offs[b - 1], offs[b]
        rows = np.arange(s - n0, e - n0)
        nb = nbrs[rows]
        joint = np.concatenate([pts[nb], pts[s:e][:, None, :]], axis=1)
        R = orf.pairwise_distances(joint, joint)
        K = orf.cov_lookup(R, bins, vals)
        L = np.linalg.cholesky(K)
        L11 = L[:, :k, :k]
        l21 = L[:, k, :k]
        sig = L[:, k, k]
        vN = values[nb]
        z = np.linalg.solve(L11, vN[..., None])[..., 0]
        w = np.linalg.solve(np.transpose(L11, (0, 2, 1)), l21[..., None])[..., 0]
        a = np.linalg.solve(np.transpose(L11, (0, 2, 1)), z[..., None])[..., 0]
        mb = vbar[s:e]
        sb = mb * xi_g[s:e] + g_logdet / sig
        grad_xi_g[s:e] = sig * mb
        np.add.at(vbar, nb, w * mb[:, None])
        # neighbour-neighbour block (ordered pairs; the a<->b symmetry is in the formula below)
        CNN = -mb[:, None, None] * (w[:, :, None] * a[:, None, :]) + (sb / sig)[:, None, None] * 0.5 * (
            w[:, :, None] * w[:, None, :])
        # d/d f(r_ab) over ordered (a, b), a != b: -mb w_a a_b + sb w_a w_b / (2 sig) each, the two orders
        # summing to the unordered derivative; diagonal: -mb w_a a_a + sb w_a^2 / (2 sig)
        _scatter_table(grad_vals, R[:, :k, :k], CNN, bins)
        cself = mb[:, None] * a - (sb / sig)[:, None] * w
        _scatter_table(grad_vals, R[:, :k, k], cself, bins)
        _scatter_table(grad_vals, R[:, k, k], sb / (2 * sig), bins)
    # dense root
    K0 = orf.compute_cov_matrix((bins, vals), pts[:n0], pts[:n0])
    L0 = np.linalg.cholesky(K0)
    y = L0.T @ vbar[:n0]
    grad_xi_g[:n0] = y
    Q = np.tril(np.outer(y, xi_g[:n0]))
    Q[np.diag_indices(n0)] *= 0.5
    Q += 0.5 * g_logdet * np.eye(n0)
    Linv = np.linalg.inv(L0)
    Kbar = Linv.T @ Q @ Linv
    _scatter_table(grad_vals, orf.pairwise_distances(pts[:n0], pts[:n0]), Kbar, bins)
    grad_xi = np.empty(n)
    grad_xi[idx] = grad_xi_g
    return grad_xi, grad_vals


def loss(graph, covariance, xi, g_values, g_logdet=0.0):
    """<g_values, generate(xi)> + g_logdet * generate_logdet: the scalar whose gradient generate_vjp returns."""
    v = orf.generate(graph, covariance, xi)
    out = float(np.dot(np.asarray(g_values, np.float64), v))
    if g_logdet:
        out += g_logdet * orf.generate_logdet(graph, covariance)
    return out
