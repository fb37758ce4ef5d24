"""Oracle: discretised kernel tables (restates reference ``graphgp/extras.py``).

Test infrastructure only; see ``oracle/__init__.py``. Tables are returned in float64; callers cast.
"""
from __future__ import annotations

import numpy as np
from scipy.special import gammaln


def make_cov_bins(*, r_min, r_max, n_bins):
    """``make_cov_bins`` (extras.py:65-68): 0 followed by n_bins-1 log-spaced radii."""
    bins = np.logspace(np.log10(r_min), np.log10(r_max), n_bins - 1)
    return np.concatenate(([0.0], bins))


def rbf_kernel(*, variance, scale, r_min, r_max, n_bins, jitter=0.0):
    """``rbf_kernel`` (extras.py:14-31)."""
    r = make_cov_bins(r_min=r_min, r_max=r_max, n_bins=n_bins)
    cov = variance * np.exp(-0.5 * (r / scale) ** 2)
    cov = np.where(r == 0.0, cov[0] * (1.0 + jitter), cov)
    return r, cov


def matern_kernel(*, p, variance, cutoff, r_min, r_max, n_bins, jitter=0.0):
    """``matern_kernel`` (extras.py:34-58): Matern nu = p + 1/2."""
    r = make_cov_bins(r_min=r_min, r_max=r_max, n_bins=n_bins)
    x = np.sqrt(2 * p + 1) * r / cutoff
    i = np.arange(p + 1)
    lf = lambda v: gammaln(np.asarray(v, dtype=np.float64) + 1)  # noqa: E731
    log_coeff = lf(p) + lf(p + i) - lf(i) - lf(p - i) - lf(2 * p)
    polynomial = np.polyval(np.exp(log_coeff), 2 * x)
    cov = variance * np.exp(-x) * polynomial
    cov = np.where(r == 0.0, cov[0] * (1.0 + jitter), cov)
    return r, cov
