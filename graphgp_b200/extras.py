"""Discretised covariance tables (host-side inputs), the same builders as reference graphgp/extras.py.

``rbf_kernel`` (extras.py:14-31), ``matern_kernel`` (Matern nu = p + 1/2, extras.py:34-58) and
``make_cov_bins`` (extras.py:65-68): r = 0 followed by ``n_bins - 1`` log-spaced radii on [r_min, r_max],
k(0) inflated by (1 + jitter). Tables are built in float64 on the host (NumPy) and returned as
``(cov_bins, cov_vals)`` arrays; pass ``device=`` to get CUDA tensors of ``dtype`` directly.
"""
from __future__ import annotations

import math

import numpy as np


def make_cov_bins(*, r_min: float, r_max: float, n_bins: int) -> np.ndarray:
    bins = np.logspace(np.log10(r_min), np.log10(r_max), n_bins - 1)
    return np.concatenate(([0.0], bins))


def _out(r, cov, device, dtype):
    if device is None:
        return r, cov
    import torch

    dtype = dtype or torch.float32
    return (torch.as_tensor(r, dtype=dtype, device=device), torch.as_tensor(cov, dtype=dtype, device=device))


def rbf_kernel(*, variance: float, scale: float, r_min: float, r_max: float, n_bins: int, jitter: float = 0.0,
               device=None, dtype=None):
    """Radial basis function (squared exponential) covariance on 0 + log-spaced bins."""
    r = make_cov_bins(r_min=r_min, r_max=r_max, n_bins=n_bins)
    cov = variance * np.exp(-0.5 * (r / scale) ** 2)
    cov = np.where(r == 0.0, cov[0] * (1.0 + jitter), cov)
    return _out(r, cov, device, dtype)


def matern_kernel(*, p: int, variance: float, cutoff: float, r_min: float, r_max: float, n_bins: int,
                  jitter: float = 0.0, device=None, dtype=None):
    """Matern covariance for nu = p + 1/2 on 0 + log-spaced bins."""
    r = make_cov_bins(r_min=r_min, r_max=r_max, n_bins=n_bins)
    x = np.sqrt(2 * p + 1) * r / cutoff
    lf = lambda v: math.lgamma(v + 1)  # noqa: E731  log factorial
    coeff = [math.exp(lf(p) + lf(p + i) - lf(i) - lf(p - i) - lf(2 * p)) for i in range(p + 1)]
    cov = variance * np.exp(-x) * np.polyval(coeff, 2 * x)
    cov = np.where(r == 0.0, cov[0] * (1.0 + jitter), cov)
    return _out(r, cov, device, dtype)
