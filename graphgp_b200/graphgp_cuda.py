"""The native boundary: the nine functions the reference calls as ``graphgp_cuda.<fn>`` behind ``cuda=True``
(graphgp/tree.py:37,61,73; graphgp/graph.py:89,106,128; graphgp/refine.py:119,216,265), with the same names,
argument meaning and results, taking and returning CUDA ``torch.Tensor`` s instead of JAX arrays.

Each call allocates its outputs and a workspace on the tensors' device and enqueues the CUDA kernels on the
current torch stream through the C ABI (include/graphgp_b200.h). Shapes are checked on the host before
launch; device-side failures surface as NaN outputs (reference refine.py:55, 182) and in the status block,
which ``last_status()`` reads back.

Beyond the nine names this module also exposes the fused whole-graph operations (``generate``,
``generate_inv``, ``generate_logdet``), the FP64 dense root (``dense``) and the adjoint (``generate_vjp``).
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

import torch

from . import _lib

DEFAULT_TAU = 1e-5
"""generate and log-determinant: FP32 points whose smallest Cholesky pivot ratio (Schur complement / prior variance)
falls below this threshold are re-conditioned in FP64 (``GGP_DEFAULT_TAU``)."""

DEFAULT_TAU_INVERSE = 3e-3
"""inverse: the same rule with a larger threshold (``GGP_DEFAULT_TAU_INVERSE``). xi = (v - mean) / std divides the
FP32 rounding of the mean by std, so the inverse needs FP64 wherever a pivot ratio is small; for k <= 20 and
d in {2, 3} an FP64 second pass finishes those points. ``tau=None`` picks each operation's default."""


def _tau(tau):
    return -1.0 if tau is None else float(tau)

_tls = threading.local()


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _suffix(dtype):
    if dtype == torch.float32:
        return "f32"
    if dtype == torch.float64:
        return "f64"
    raise TypeError(f"points / values must be float32 or float64, got {dtype}")


def _cuda(t, name, dtype=None):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (this package has no CPU path)")
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def _ids(t, name):
    return _cuda(t, name, torch.int32)


def _workspace(op, n, d, n0, k, nb, n_off, tbytes, device):
    lib = _lib.load()
    size = lib.ggp_workspace_size(_lib.OPS[op], int(n), int(d), int(n0), int(k), int(nb), int(n_off), int(tbytes))
    ws = torch.empty(max(size, 256), dtype=torch.uint8, device=device)
    _tls.last_ws = ws
    return ws


def last_status():
    """Status block of the most recent call on this thread (synchronises the current stream)."""
    ws = getattr(_tls, "last_ws", None)
    if ws is None:
        return None
    st = _lib.Status()
    _lib.check(_lib.load().ggp_read_status(_ptr(ws), C.byref(st), _stream()), "ggp_read_status")
    return dict(error=st.error, nan_seen=st.nan_seen, fallback_count=st.fallback_count, timeouts=st.timeouts)


def _table(cov_bins, cov_vals, dtype):
    bins = _cuda(cov_bins, "cov_bins", dtype)
    vals = _cuda(cov_vals, "cov_vals", dtype)
    if bins.ndim != 1 or vals.shape != bins.shape or len(bins) < 2:
        raise ValueError("cov_bins and cov_vals must be 1-D arrays of equal length >= 2")
    return bins, vals


def _offsets(offsets, device):
    if isinstance(offsets, torch.Tensor):
        return _ids(offsets.to(device), "offsets")
    return torch.as_tensor(list(offsets), dtype=torch.int32, device=device)


# ------------------------------------------------------------------------------------------------
# graph build (reference graphgp/tree.py, graphgp/graph.py)
# ------------------------------------------------------------------------------------------------
def build_tree(points):
    """``graphgp_cuda.build_tree(points)`` (tree.py:37) -> (points_tree, split_dims, indices)."""
    points = _cuda(points, "points")
    if points.ndim != 2:
        raise ValueError(f"Points must have shape (N, d). Got shape {tuple(points.shape)}.")
    sfx = _suffix(points.dtype)
    n, d = points.shape
    out_p = torch.empty_like(points)
    split = torch.empty(n, dtype=torch.int32, device=points.device)
    idx = torch.empty(n, dtype=torch.int32, device=points.device)
    ws = _workspace("BUILD_TREE", n, d, 0, 0, 2, 1, points.element_size(), points.device)
    fn = getattr(_lib.load(), f"ggp_build_tree_{sfx}")
    _lib.check(fn(_ptr(points), n, d, _ptr(out_p), _ptr(split), _ptr(idx), _ptr(ws), ws.numel(), _stream()),
               "build_tree")
    return out_p, split, idx


def query_neighbors(points, split_dims, query_indices, max_indices, *, k):
    """``graphgp_cuda.query_neighbors`` (tree.py:73): k nearest among tree nodes < max_indices[q]."""
    points = _cuda(points, "points")
    sfx = _suffix(points.dtype)
    split_dims = _ids(split_dims, "split_dims")
    q = _ids(query_indices, "query_indices")
    m = _ids(max_indices, "max_indices")
    n, d = points.shape
    nq = q.numel()
    if m.numel() != nq:
        raise ValueError("query_indices and max_indices must have the same length")
    out = torch.empty((nq, k), dtype=torch.int32, device=points.device)
    ws = _workspace("QUERY_NEIGHBORS", n, d, 0, k, 2, 1, points.element_size(), points.device)
    fn = getattr(_lib.load(), f"ggp_query_neighbors_{sfx}")
    _lib.check(fn(_ptr(points), _ptr(split_dims), n, d, _ptr(q), _ptr(m), nq, int(k), _ptr(out), _ptr(ws),
                  ws.numel(), _stream()), "query_neighbors")
    return out


def query_preceding_neighbors(points, split_dims, *, n0, k):
    """``graphgp_cuda.query_preceding_neighbors`` (tree.py:61): k nearest preceding points for rows >= n0."""
    if n0 < k:
        raise ValueError(f"n0 must be at least k. Got n0={n0}, k={k}.")
    points = _cuda(points, "points")
    sfx = _suffix(points.dtype)
    split_dims = _ids(split_dims, "split_dims")
    n, d = points.shape
    out = torch.empty((n - n0, k), dtype=torch.int32, device=points.device)
    ws = _workspace("QUERY_NEIGHBORS", n, d, n0, k, 2, 1, points.element_size(), points.device)
    fn = getattr(_lib.load(), f"ggp_query_preceding_neighbors_{sfx}")
    _lib.check(fn(_ptr(points), _ptr(split_dims), n, d, int(n0), int(k), _ptr(out), _ptr(ws), ws.numel(),
                  _stream()), "query_preceding_neighbors")
    return out


def compute_depths_parallel(neighbors, *, n0):
    """``graphgp_cuda.compute_depths_parallel(neighbors, n0=)`` (graph.py:106)."""
    nb = _ids(neighbors, "neighbors")
    rows, k = nb.shape
    n = n0 + rows
    out = torch.empty(n, dtype=torch.int32, device=nb.device)
    ws = _workspace("COMPUTE_DEPTHS", n, 1, n0, k, 2, 1, 4, nb.device)
    _lib.check(_lib.load().ggp_compute_depths(_ptr(nb), n, int(n0), k, _ptr(out), _ptr(ws), ws.numel(), _stream()),
               "compute_depths")
    return out


def order_by_depth(points, indices, neighbors, depths, *, return_offsets=False):
    """``graphgp_cuda.order_by_depth(points, indices, neighbors, depths)`` (graph.py:128).

    With ``return_offsets=True`` also returns the batch offsets (graph.py:95-96) as a host tuple."""
    points = _cuda(points, "points")
    sfx = _suffix(points.dtype)
    indices = _ids(indices, "indices")
    nb = _ids(neighbors, "neighbors")
    depths = _ids(depths, "depths")
    n, d = points.shape
    rows, k = nb.shape
    n0 = n - rows
    outs = (torch.empty_like(points), torch.empty_like(indices), torch.empty_like(nb), torch.empty_like(depths))
    offs = torch.empty(n + 1, dtype=torch.int32, device=points.device)
    n_off = torch.empty(1, dtype=torch.int32, device=points.device)
    ws = _workspace("ORDER_BY_DEPTH", n, d, n0, k, 2, 1, points.element_size(), points.device)
    fn = getattr(_lib.load(), f"ggp_order_by_depth_{sfx}")
    _lib.check(fn(_ptr(points), _ptr(indices), _ptr(nb), _ptr(depths), n, d, n0, k, *map(_ptr, outs), _ptr(offs),
                  _ptr(n_off), _ptr(ws), ws.numel(), _stream()), "order_by_depth")
    if return_offsets:
        cnt = int(n_off.item())
        return (*outs, tuple(int(x) for x in offs[:cnt].tolist()))
    return outs


def build_graph(points, *, n0, k, return_offsets=False):
    """``graphgp_cuda.build_graph(points, n0=, k=)`` (graph.py:89) -> (points, indices, neighbors, depths)."""
    if n0 < k:
        raise ValueError(f"n0 must be at least k. Got n0={n0}, k={k}.")
    points = _cuda(points, "points")
    if points.ndim != 2:
        raise ValueError(f"Points must have shape (N, d). Got shape {tuple(points.shape)}.")
    sfx = _suffix(points.dtype)
    n, d = points.shape
    if n0 > n:
        raise ValueError("n0 must not exceed the number of points")
    dev = points.device
    out_p = torch.empty_like(points)
    idx = torch.empty(n, dtype=torch.int32, device=dev)
    nbrs = torch.empty((n - n0, k), dtype=torch.int32, device=dev)
    depths = torch.empty(n, dtype=torch.int32, device=dev)
    offs = torch.empty(n + 1, dtype=torch.int32, device=dev)
    n_off = torch.empty(1, dtype=torch.int32, device=dev)
    ws = _workspace("BUILD_GRAPH", n, d, n0, k, 2, 1, points.element_size(), dev)
    fn = getattr(_lib.load(), f"ggp_build_graph_{sfx}")
    _lib.check(fn(_ptr(points), n, d, int(n0), int(k), _ptr(out_p), _ptr(idx), _ptr(nbrs), _ptr(depths), _ptr(offs),
                  _ptr(n_off), _ptr(ws), ws.numel(), _stream()), "build_graph")
    if return_offsets:
        cnt = int(n_off.item())
        return out_p, idx, nbrs, depths, tuple(int(x) for x in offs[:cnt].tolist())
    return out_p, idx, nbrs, depths


# ------------------------------------------------------------------------------------------------
# refinement (reference graphgp/refine.py)
# ------------------------------------------------------------------------------------------------
def _refine_common(points, neighbors, offsets):
    points = _cuda(points, "points")
    sfx = _suffix(points.dtype)
    nb = _ids(neighbors, "neighbors")
    if nb.ndim != 2:
        raise ValueError("neighbors must have shape (N - n0, k)")
    n, d = points.shape
    rows, k = nb.shape
    n0 = n - rows
    offs = _offsets(offsets, points.device)
    return points, sfx, nb, n, d, n0, k, offs


def refine(points, neighbors, offsets, cov_bins, cov_vals, initial_values, xi, *, tau=None, timeout_ns=0):
    """``graphgp_cuda.refine`` (refine.py:119-121): values (N,) in graph order."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    init = _cuda(initial_values, "initial_values", points.dtype)
    xi = _cuda(xi, "xi", points.dtype)
    if init.numel() != n0:
        raise ValueError("Length of initial_values must match number of initial points.")
    if xi.numel() != n - n0:
        raise ValueError("Length of xi must match number of refined points.")
    out = torch.empty(n, dtype=points.dtype, device=points.device)
    ws = _workspace("REFINE", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_refine_f32(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins), _ptr(vals),
                                len(bins), _ptr(init), _ptr(xi), _ptr(out), _tau(tau), int(timeout_ns), _ptr(ws),
                                ws.numel(), _stream())
    else:
        rc = lib.ggp_refine_f64(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins), _ptr(vals),
                                len(bins), _ptr(init), _ptr(xi), _ptr(out), int(timeout_ns), _ptr(ws), ws.numel(),
                                _stream())
    _lib.check(rc, "refine")
    return out


def refine_inv(points, neighbors, offsets, cov_bins, cov_vals, values, *, tau=None):
    """``graphgp_cuda.refine_inv`` (refine.py:216-218) -> (initial_values (n0,), xi (N - n0,))."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    values = _cuda(values, "values", points.dtype)
    if values.numel() != n:
        raise ValueError("Length of values must match number of points.")
    init = torch.empty(n0, dtype=points.dtype, device=points.device)
    xi = torch.empty(n - n0, dtype=points.dtype, device=points.device)
    ws = _workspace("REFINE_INV", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_refine_inv_f32(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                    _ptr(vals), len(bins), _ptr(values), _ptr(init), _ptr(xi), _tau(tau), _ptr(ws),
                                    ws.numel(), _stream())
    else:
        rc = lib.ggp_refine_inv_f64(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                    _ptr(vals), len(bins), _ptr(values), _ptr(init), _ptr(xi), _ptr(ws), ws.numel(),
                                    _stream())
    _lib.check(rc, "refine_inv")
    return init, xi


def refine_logdet(points, neighbors, offsets, cov_bins, cov_vals, *, tau=None):
    """``graphgp_cuda.refine_logdet`` (refine.py:265): sum of log std, FP64 accumulation (0-d float64 tensor)."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    out = torch.empty((), dtype=torch.float64, device=points.device)
    ws = _workspace("REFINE_LOGDET", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_refine_logdet_f32(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                       _ptr(vals), len(bins), _ptr(out), _tau(tau), _ptr(ws), ws.numel(), _stream())
    else:
        rc = lib.ggp_refine_logdet_f64(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                       _ptr(vals), len(bins), _ptr(out), _ptr(ws), ws.numel(), _stream())
    _lib.check(rc, "refine_logdet")
    return out


# ------------------------------------------------------------------------------------------------
# FP64 dense root and fused whole-graph operations
# ------------------------------------------------------------------------------------------------
def dense(mode, points, cov_bins, cov_vals, x=None):
    """FP64 dense root on ``points`` (n0, d): mode "generate" -> L @ x, "inverse" -> L^-1 x, "logdet" ->
    sum log L_ii = slogdet(K)/2 (reference refine.py:59-76, 186-195, 243-248)."""
    points = _cuda(points, "points")
    sfx = _suffix(points.dtype)
    n0, d = points.shape
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    m = {"generate": 0, "inverse": 1, "logdet": 2}[mode]
    x = None if x is None else _cuda(x, "x", points.dtype)
    if m < 2 and (x is None or x.numel() != n0):
        raise ValueError("Length of xi / values must match number of points.")
    out = torch.empty(n0, dtype=points.dtype, device=points.device) if m < 2 else None
    ld = torch.empty((), dtype=torch.float64, device=points.device) if m == 2 else None
    ws = _workspace("DENSE", n0, d, n0, 1, len(bins), 1, points.element_size(), points.device)
    fn = getattr(_lib.load(), f"ggp_dense_{sfx}")
    _lib.check(fn(m, _ptr(points), n0, d, _ptr(bins), _ptr(vals), len(bins), _ptr(x), _ptr(out), _ptr(ld), _ptr(ws),
                  ws.numel(), _stream()), "dense")
    return out if m < 2 else ld


def generate(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, *, tau=None, timeout_ns=0):
    """Whole ``generate`` (reference refine.py:21-56) in one device call: xi (N,) in the original order ->
    values (N,) in the original order; ``indices`` may be None."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    xi = _cuda(xi, "xi", points.dtype)
    if xi.numel() != n:
        raise ValueError("Length of xi must match number of points in graph.")
    idx = None if indices is None else _ids(indices, "indices")
    out = torch.empty(n, dtype=points.dtype, device=points.device)
    ws = _workspace("GENERATE", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_generate_f32(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                  _ptr(vals), len(bins), _ptr(xi), _ptr(out), _tau(tau), int(timeout_ns), _ptr(ws),
                                  ws.numel(), _stream())
    else:
        rc = lib.ggp_generate_f64(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                  _ptr(vals), len(bins), _ptr(xi), _ptr(out), int(timeout_ns), _ptr(ws), ws.numel(),
                                  _stream())
    _lib.check(rc, "generate")
    return out


def generate_and_logdet(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, *, tau=None, timeout_ns=0,
                        with_resid=False):
    """``generate`` and ``generate_logdet`` of the same table -> (values (N,), logdet (0-d float64)). In FP32 one
    pass computes both (``ggp_generate_and_logdet_f32``); in FP64 the two calls run one after the other.

    ``with_resid``: also return the adjoint's residuals ((N - n0) x (2k + 1) FP32, for ``generate_vjp(resid=...)``)
    as a third element, or None where the pass does not write them (FP64, k > 20, d not in {2, 3})."""
    if _suffix(_cuda(points, "points").dtype) != "f32":
        out = (generate(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, tau=tau, timeout_ns=timeout_ns),
               generate_logdet(points, neighbors, offsets, cov_bins, cov_vals, tau=tau))
        return out + (None,) if with_resid else out
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    xi = _cuda(xi, "xi", points.dtype)
    if xi.numel() != n:
        raise ValueError("Length of xi must match number of points in graph.")
    idx = None if indices is None else _ids(indices, "indices")
    out = torch.empty(n, dtype=points.dtype, device=points.device)
    ld = torch.empty((), dtype=torch.float64, device=points.device)
    ws = _workspace("GENERATE", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    resid = None
    written = C.c_int(0)
    if with_resid and n > n0 and k <= 20 and d in (2, 3):
        resid = torch.empty((n - n0, 2 * k + 1), dtype=torch.float32, device=points.device)
    rc = _lib.load().ggp_generate_and_logdet_f32(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                                 _ptr(bins), _ptr(vals), len(bins), _ptr(xi), _ptr(out), _ptr(ld),
                                                 _ptr(resid), C.byref(written), _tau(tau), int(timeout_ns),
                                                 _ptr(ws), ws.numel(), _stream())
    _lib.check(rc, "generate_and_logdet")
    if not with_resid:
        return out, ld
    return out, ld, (resid if written.value else None)


def generate_inv(points, indices, neighbors, offsets, cov_bins, cov_vals, values, *, tau=None):
    """Whole ``generate_inv`` (reference refine.py:162-183) in one device call."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    values = _cuda(values, "values", points.dtype)
    if values.numel() != n:
        raise ValueError("Length of values must match number of points in graph.")
    idx = None if indices is None else _ids(indices, "indices")
    out = torch.empty(n, dtype=points.dtype, device=points.device)
    ws = _workspace("GENERATE_INV", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_generate_inv_f32(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                      _ptr(bins), _ptr(vals), len(bins), _ptr(values), _ptr(out), _tau(tau), _ptr(ws),
                                      ws.numel(), _stream())
    else:
        rc = lib.ggp_generate_inv_f64(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                      _ptr(bins), _ptr(vals), len(bins), _ptr(values), _ptr(out), _ptr(ws), ws.numel(),
                                      _stream())
    _lib.check(rc, "generate_inv")
    return out


def generate_logdet(points, neighbors, offsets, cov_bins, cov_vals, *, tau=None):
    """Whole ``generate_logdet`` (reference refine.py:234-240): dense + refined, 0-d float64 tensor."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    out = torch.empty((), dtype=torch.float64, device=points.device)
    ws = _workspace("GENERATE_LOGDET", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if sfx == "f32":
        rc = lib.ggp_generate_logdet_f32(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                         _ptr(vals), len(bins), _ptr(out), _tau(tau), _ptr(ws), ws.numel(), _stream())
    else:
        rc = lib.ggp_generate_logdet_f64(_ptr(points), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs), _ptr(bins),
                                         _ptr(vals), len(bins), _ptr(out), _ptr(ws), ws.numel(), _stream())
    _lib.check(rc, "generate_logdet")
    return out


def generate_vjp(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, g_values, g_logdet=0.0, *,
                 tau=None, values=None, resid=None):
    """Adjoint of generate (+ g_logdet * generate_logdet): returns (grad_xi (N,), grad_cov_vals (n_bins,) f64).

    ``values``: generate's output for these same inputs, if the caller has it (the primal output a custom_vjp
    keeps); it saves recomputing the forward pass. ``resid``: the residuals ``generate_and_logdet(with_resid=True)``
    returned for the same inputs (FP32, needs ``values``); the reverse sweep then reads each row's w, a and sigma
    instead of refactorising it. Without them the per-point factorisations are recomputed."""
    points, sfx, nb, n, d, n0, k, offs = _refine_common(points, neighbors, offsets)
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    xi = _cuda(xi, "xi", points.dtype)
    g = _cuda(g_values, "g_values", points.dtype)
    if xi.numel() != n or g.numel() != n:
        raise ValueError("xi and g_values must have one entry per point")
    idx = None if indices is None else _ids(indices, "indices")
    if values is not None:
        values = _cuda(values, "values", points.dtype)
        if values.numel() != n:
            raise ValueError("values must have one entry per point")
    gx = torch.empty(n, dtype=points.dtype, device=points.device)
    gv = torch.empty(len(bins), dtype=torch.float64, device=points.device)
    ws = _workspace("GENERATE_VJP", n, d, n0, k, len(bins), len(offs), points.element_size(), points.device)
    lib = _lib.load()
    if resid is not None:
        if sfx != "f32" or values is None:
            raise ValueError("resid needs FP32 inputs and values")
        resid = _cuda(resid, "resid", torch.float32)
        if resid.numel() != (n - n0) * (2 * k + 1):
            raise ValueError("resid must hold (N - n0) x (2k + 1) entries")
        rc = lib.ggp_generate_vjp_resid_f32(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                            _ptr(bins), _ptr(vals), len(bins), _ptr(xi), _ptr(values), _ptr(resid),
                                            _ptr(g), float(g_logdet), _ptr(gx), _ptr(gv), _tau(tau), _ptr(ws),
                                            ws.numel(), _stream())
    elif sfx == "f32":
        rc = lib.ggp_generate_vjp_f32(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                      _ptr(bins), _ptr(vals), len(bins), _ptr(xi), _ptr(values), _ptr(g),
                                      float(g_logdet), _ptr(gx),
                                      _ptr(gv), _tau(tau), _ptr(ws), ws.numel(), _stream())
    else:
        rc = lib.ggp_generate_vjp_f64(_ptr(points), _ptr(idx), n, d, n0, _ptr(nb), k, _ptr(offs), len(offs),
                                      _ptr(bins), _ptr(vals), len(bins), _ptr(xi), _ptr(values), _ptr(g),
                                      float(g_logdet), _ptr(gx),
                                      _ptr(gv), _ptr(ws), ws.numel(), _stream())
    _lib.check(rc, "generate_vjp")
    return gx, gv


_REQUEST_OPS = {"generate": 0, "inverse": 1, "logdet": 2}


def request(op, points, n0, k, cov_bins, cov_vals, payload=None, *, tau=None):
    """Graph build plus one operation in a single native call (``ggp_request_*``): op "generate" (payload = xi)
    or "inverse" (payload = values) -> (N,) tensor in the caller's order; "logdet" -> 0-d float64 tensor. Builds
    the same graph as ``build_graph(points, n0=n0, k=k)``; the call waits on the current stream once."""
    if op not in _REQUEST_OPS:
        raise ValueError(f"unknown op {op!r}")
    if n0 < k:
        raise ValueError(f"n0 must be at least k. Got n0={n0}, k={k}.")
    points = _cuda(points, "points")
    if points.ndim != 2:
        raise ValueError(f"Points must have shape (N, d). Got shape {tuple(points.shape)}.")
    sfx = _suffix(points.dtype)
    n, d = points.shape
    if n0 > n:
        raise ValueError("n0 must not exceed the number of points")
    bins, vals = _table(cov_bins, cov_vals, points.dtype)
    m = _REQUEST_OPS[op]
    lib = _lib.load()
    out = ld = None
    if m < 2:
        payload = _cuda(payload, "payload", points.dtype)
        if payload.numel() != n:
            raise ValueError("payload must have one entry per point")
        out = torch.empty(n, dtype=points.dtype, device=points.device)
    else:
        ld = torch.empty((), dtype=torch.float64, device=points.device)
    size = lib.ggp_request_buffer_size(m, n, d, int(n0), int(k), len(bins), points.element_size())
    buf = torch.empty(max(size, 256), dtype=torch.uint8, device=points.device)
    _tls.last_ws = buf
    if sfx == "f32":
        rc = lib.ggp_request_f32(m, _ptr(points), n, d, int(n0), int(k), _ptr(bins), _ptr(vals), len(bins),
                                 _ptr(payload if m < 2 else None), _ptr(out), _ptr(ld), _tau(tau), _ptr(buf),
                                 buf.numel(), _stream())
    else:
        rc = lib.ggp_request_f64(m, _ptr(points), n, d, int(n0), int(k), _ptr(bins), _ptr(vals), len(bins),
                                 _ptr(payload if m < 2 else None), _ptr(out), _ptr(ld), _ptr(buf), buf.numel(),
                                 _stream())
    _lib.check(rc, "request")
    return out if m < 2 else ld


def request_host(op, points, n0, k, cov_bins, cov_vals, payload=None, *, tau=None, buffers=None, device=None):
    """``request`` with host (numpy) arrays end to end (``ggp_request_host_*``): the inputs go up through a pinned
    staging block in one copy, the graph build and operation run on the current stream, and the result and the
    status block come back before the call returns, all inside one native call. Returns (output, status dict):
    output is the (N,) numpy array in the caller's order, or the float log-determinant. ``buffers`` (a dict)
    keeps the device and pinned blocks between calls, grown when a request needs more."""
    if op not in _REQUEST_OPS:
        raise ValueError(f"unknown op {op!r}")
    if n0 < k:
        raise ValueError(f"n0 must be at least k. Got n0={n0}, k={k}.")
    pts = np.asarray(points)
    if pts.ndim != 2:
        raise ValueError(f"Points must have shape (N, d). Got shape {tuple(pts.shape)}.")
    dt = np.float64 if pts.dtype == np.float64 else np.float32
    pts = np.ascontiguousarray(pts, dt)
    n, d = pts.shape
    if n0 > n:
        raise ValueError("n0 must not exceed the number of points")
    bins = np.ascontiguousarray(cov_bins, dt)
    vals = np.ascontiguousarray(cov_vals, dt)
    if bins.ndim != 1 or vals.shape != bins.shape or len(bins) < 2:
        raise ValueError("cov_bins and cov_vals must be 1-D arrays of equal length >= 2")
    m = _REQUEST_OPS[op]
    x = None
    out = None
    if m < 2:
        x = np.ascontiguousarray(payload, dt).reshape(-1)
        if x.size != n:
            raise ValueError("payload must have one entry per point")
        out = np.empty(n, dt)
    lib = _lib.load()
    dev_b, pin_b = C.c_size_t(), C.c_size_t()
    _lib.check(lib.ggp_request_host_sizes(m, n, d, int(n0), int(k), len(bins), np.dtype(dt).itemsize,
                                          C.byref(dev_b), C.byref(pin_b)), "request_host")
    buffers = {} if buffers is None else buffers
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    dbuf = buffers.get("device")
    if dbuf is None or dbuf.numel() < dev_b.value or dbuf.device != device:
        dbuf = buffers["device"] = torch.empty(max(dev_b.value, 1 << 20), dtype=torch.uint8, device=device)
    pbuf = buffers.get("pinned")
    if pbuf is None or pbuf.numel() < pin_b.value:
        pbuf = buffers["pinned"] = torch.empty(max(pin_b.value, 1 << 20), dtype=torch.uint8, pin_memory=True)
    _tls.last_ws = dbuf
    ld = C.c_double(0.0)
    st = _lib.Status()
    addr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    if dt == np.float32:
        rc = lib.ggp_request_host_f32(m, addr(pts), n, d, int(n0), int(k), addr(bins), addr(vals), len(bins), addr(x),
                                      addr(out), C.byref(ld), C.byref(st), _tau(tau), dbuf.data_ptr(), dbuf.numel(),
                                      pbuf.data_ptr(), pbuf.numel(), _stream())
    else:
        rc = lib.ggp_request_host_f64(m, addr(pts), n, d, int(n0), int(k), addr(bins), addr(vals), len(bins), addr(x),
                                      addr(out), C.byref(ld), C.byref(st), dbuf.data_ptr(), dbuf.numel(),
                                      pbuf.data_ptr(), pbuf.numel(), _stream())
    _lib.check(rc, "request_host")
    status = dict(error=st.error, nan_seen=st.nan_seen, fallback_count=st.fallback_count, timeouts=st.timeouts)
    return (out if m < 2 else float(ld.value)), status


def wait_probe(timeout_ns=1_000_000):
    """Run the bounded-wait probe kernel; returns the status code it observed (GGP_ERR_TIMEOUT expected)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    ws = torch.empty(512, dtype=torch.uint8, device=dev)
    code = C.c_int(-1)
    _lib.check(_lib.load().ggp_wait_probe(int(timeout_ns), C.byref(code), _ptr(ws), ws.numel(), _stream()),
               "wait_probe")
    return code.value
