"""Test helpers: seeded synthetic inputs and oracle-built graphs (test infrastructure)."""
from __future__ import annotations

import functools

import numpy as np

from oracle import extras as ox
from oracle import graph as og


@functools.lru_cache(maxsize=None)
def oracle_graph(n, d, n0, k, seed=0, dtype="float32", dist="normal"):
    rng = np.random.default_rng(seed)
    if dist == "normal":
        pts = rng.standard_normal((n, d))
    elif dist == "uniform":
        pts = rng.uniform(0, 1, (n, d))
    elif dist == "shell":  # unit direction times radius 10^U(-3, 0), heavy dynamic range
        v = rng.standard_normal((n, d))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pts = v * 10.0 ** rng.uniform(-3, 0, (n, 1))
    else:
        raise ValueError(dist)
    pts = pts.astype(dtype)
    return pts, og.build_graph(pts, n0=n0, k=k)


def rbf_table(scale=0.3, r_min=1e-4, r_max=10.0, n_bins=1001, jitter=1e-4):
    return ox.rbf_kernel(variance=1.0, scale=scale, r_min=r_min, r_max=r_max, n_bins=n_bins, jitter=jitter)


def matern32_table(cutoff=0.05, r_min=1e-6, r_max=4.0, n_bins=2049, jitter=1e-5):
    return ox.matern_kernel(p=1, variance=1.0, cutoff=cutoff, r_min=r_min, r_max=r_max, n_bins=n_bins, jitter=jitter)


def as_inputs(cov, dtype):
    """The table as a kernel of that dtype receives it: rounded to `dtype`, held in float64 for the oracle. FP32
    results are compared with the FP64 oracle on these same inputs, so that the error measured is the FP32
    arithmetic's, not the rounding of the caller's table (which alone moves a smooth-kernel inverse by ~2e-4)."""
    bins, vals = cov
    return (np.asarray(bins).astype(dtype).astype(np.float64), np.asarray(vals).astype(dtype).astype(np.float64))
