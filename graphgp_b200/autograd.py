"""Differentiable ``generate`` and ``generate_logdet``: ``torch.autograd.Function`` s whose backward passes call the
hand-written adjoint kernels (``ggp_generate_vjp_*``, include/graphgp_b200.h).

The reference differentiates ``generate`` with JAX autodiff (graphgp/refine.py:21-56 through 123-145; its tests
take ``jax.jacfwd`` of it, tests/test_refine.py:77), and its README promises the CUDA primitives' derivatives with
respect to the white noise and the kernel parameters (README.md:36). Here the same derivatives come from one
reverse sweep on the device:

* ``GenerateFn``: values = generate(xi, cov_vals); the forward keeps ``values`` as its residual (the adjoint then
  skips recomputing the forward pass; every per-point Cholesky factor is recomputed, never stored), and the
  backward returns d<g, values>/dxi (N,) and d<g, values>/dcov_vals (n_bins,).
* ``GenerateLogdetFn``: logdet = generate_logdet(cov_vals) (FP64 0-d tensor); its backward returns
  g * dlogdet/dcov_vals through the same adjoint with a zero value cotangent.
* ``GenerateAndLogdetFn``: both at once, with one adjoint sweep for both cotangents (a Gaussian likelihood). With
  ``RESIDUALS = True`` (FP32, 10 < k <= 20, d in {2, 3}) its forward also keeps each refined row's w, a and sigma,
  which the backward sweep reads instead of refactorising the row.

The graph (points, neighbours, offsets, indices) and the table's bins are constants: no gradient flows to them.
This is the JAX ``custom_vjp`` that a ``jax.ffi`` host would register written for torch.
"""
from __future__ import annotations

import torch

from . import graphgp_cuda as _gc

# False (the default): the backward sweep recomputes every refined row's factorisation and nothing per row is kept.
# True: GenerateAndLogdetFn keeps each refined row's w, a and sigma from its forward pass ((2k + 1) FP32 per row, no
# Cholesky factor) and the backward sweep reads them instead of refactorising (FP32, 10 < k <= 20, d in {2, 3}).
RESIDUALS = False


class GenerateFn(torch.autograd.Function):
    """values = generate(points, indices, neighbors, offsets, cov_bins, cov_vals, xi), differentiable in xi and
    cov_vals."""

    @staticmethod
    def forward(ctx, xi, cov_vals, points, indices, neighbors, offsets, cov_bins, tau):
        values = _gc.generate(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, tau=tau)
        ctx.save_for_backward(xi, cov_vals, values)
        ctx.graph = (points, indices, neighbors, offsets, cov_bins, tau)
        return values

    @staticmethod
    def backward(ctx, g_values):
        xi, cov_vals, values = ctx.saved_tensors
        points, indices, neighbors, offsets, cov_bins, tau = ctx.graph
        need_xi, need_vals = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_xi or need_vals):
            return (None,) * 8
        gx, gv = _gc.generate_vjp(points, indices, neighbors, offsets, cov_bins, cov_vals, xi,
                                  g_values.to(values.dtype).contiguous(), 0.0, tau=tau, values=values)
        return (gx if need_xi else None, gv.to(cov_vals.dtype) if need_vals else None) + (None,) * 6


class GenerateLogdetFn(torch.autograd.Function):
    """logdet = generate_logdet(points, neighbors, offsets, cov_bins, cov_vals) (FP64), differentiable in
    cov_vals."""

    @staticmethod
    def forward(ctx, cov_vals, points, indices, neighbors, offsets, cov_bins, tau):
        out = _gc.generate_logdet(points, neighbors, offsets, cov_bins, cov_vals, tau=tau)
        ctx.save_for_backward(cov_vals)
        ctx.graph = (points, indices, neighbors, offsets, cov_bins)
        return out

    @staticmethod
    def backward(ctx, g):
        (cov_vals,) = ctx.saved_tensors
        if not ctx.needs_input_grad[0]:
            return (None,) * 7
        points, indices, neighbors, offsets, cov_bins = ctx.graph
        n = points.shape[0]
        zeros = torch.zeros(n, dtype=points.dtype, device=points.device)
        # a zero value cotangent leaves only the log-determinant's terms; the residual can be anything
        _, gv = _gc.generate_vjp(points, indices, neighbors, offsets, cov_bins, cov_vals, zeros, zeros,
                                 float(g), values=zeros)
        return (gv.to(cov_vals.dtype),) + (None,) * 6


class GenerateAndLogdetFn(torch.autograd.Function):
    """(values, logdet) = (generate(xi, cov_vals), generate_logdet(cov_vals)), computed in one forward pass (FP32),
    with one backward sweep for both cotangents: the adjoint takes g_values and g_logdet together, so a loss that uses both (a Gaussian likelihood:
    0.5 |values - y|^2 + logdet) costs one reverse pass instead of two."""

    @staticmethod
    def forward(ctx, xi, cov_vals, points, indices, neighbors, offsets, cov_bins, tau):
        out = _gc.generate_and_logdet(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, tau=tau,
                                      with_resid=RESIDUALS)
        values, logdet, resid = out if RESIDUALS else out + (None,)
        ctx.save_for_backward(xi, cov_vals, values, resid)
        ctx.graph = (points, indices, neighbors, offsets, cov_bins, tau)
        return values, logdet

    @staticmethod
    def backward(ctx, g_values, g_logdet):
        xi, cov_vals, values, resid = ctx.saved_tensors
        points, indices, neighbors, offsets, cov_bins, tau = ctx.graph
        need_xi, need_vals = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_xi or need_vals):
            return (None,) * 8
        if g_values is None:
            g_values = torch.zeros_like(values)
        gl = 0.0 if g_logdet is None else float(g_logdet)
        gx, gv = _gc.generate_vjp(points, indices, neighbors, offsets, cov_bins, cov_vals, xi,
                                  g_values.to(values.dtype).contiguous(), gl, tau=tau, values=values, resid=resid)
        return (gx if need_xi else None, gv.to(cov_vals.dtype) if need_vals else None) + (None,) * 6


def generate(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, *, tau=None):
    """``graphgp_cuda.generate`` recorded for autograd (xi and cov_vals may require grad)."""
    return GenerateFn.apply(xi, cov_vals, points, indices, neighbors, offsets, cov_bins, tau)


def generate_logdet(points, indices, neighbors, offsets, cov_bins, cov_vals, *, tau=None):
    """``graphgp_cuda.generate_logdet`` recorded for autograd (cov_vals may require grad)."""
    return GenerateLogdetFn.apply(cov_vals, points, indices, neighbors, offsets, cov_bins, tau)


def generate_and_logdet(points, indices, neighbors, offsets, cov_bins, cov_vals, xi, *, tau=None):
    """(values, logdet) recorded for autograd with a single adjoint sweep in the backward pass."""
    return GenerateAndLogdetFn.apply(xi, cov_vals, points, indices, neighbors, offsets, cov_bins, tau)
