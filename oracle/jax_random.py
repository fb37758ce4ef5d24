"""NumPy restatement of JAX's default PRNG (threefry2x32) for ``jax.random.key`` / ``jax.random.normal``.

Test infrastructure only (part of the oracle): it regenerates the random inputs the reference's own tests
draw with ``jr.key(137)`` (reference ``tests/test_tree.py:9``, ``tests/test_graph.py:11``,
``tests/test_refine.py:12``) so that the reference's RNG-bound golden values can pin the oracle without JAX.

Algorithm sources (published): Threefry-2x32 with 20 rounds from Salmon et al., "Parallel random numbers:
as easy as 1, 2, 3" (SC'11); JAX 0.8's key derivation (seed -> [seed >> 32, seed & 0xffffffff]), its
"partitionable" counter layout (64-bit row-major iota split into hi/lo words), its uniform construction
(random mantissa bits with exponent of 1.0, minus 1, then scale/shift and clamp) and its normal sampler
(sqrt(2) * erfinv(u), u uniform on (nextafter(-1, 0), 1)).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erfinv

_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))
_M32 = np.uint64(0xFFFFFFFF)


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return ((x << np.uint64(r)) | (x >> np.uint64(32 - r))) & _M32


def threefry2x32(k0: int, k1: int, x0: np.ndarray, x1: np.ndarray):
    """Threefry-2x32, 20 rounds, on uint32 counters (carried in uint64 to avoid overflow warnings)."""
    ks = [np.uint64(k0), np.uint64(k1), np.uint64((k0 ^ k1 ^ 0x1BD11BDA) & 0xFFFFFFFF)]
    x0 = (np.asarray(x0, np.uint64) + ks[0]) & _M32
    x1 = (np.asarray(x1, np.uint64) + ks[1]) & _M32
    for i in range(5):
        for r in _ROT[i % 2]:
            x0 = (x0 + x1) & _M32
            x1 = _rotl(x1, r) ^ x0
        x0 = (x0 + ks[(i + 1) % 3]) & _M32
        x1 = (x1 + ks[(i + 2) % 3] + np.uint64(i + 1)) & _M32
    return x0.astype(np.uint32), x1.astype(np.uint32)


def key(seed: int):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return (seed >> 32, seed & 0xFFFFFFFF)


def random_bits64(k, shape) -> np.ndarray:
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.uint64)
    hi, lo = threefry2x32(k[0], k[1], idx >> np.uint64(32), idx & _M32)
    return ((hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)).reshape(shape)


def random_bits32(k, shape) -> np.ndarray:
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.uint64)
    hi, lo = threefry2x32(k[0], k[1], idx >> np.uint64(32), idx & _M32)
    return (hi ^ lo).reshape(shape)


def uniform(k, shape, dtype=np.float64, minval=0.0, maxval=1.0) -> np.ndarray:
    dtype = np.dtype(dtype)
    if dtype == np.float64:
        bits = random_bits64(k, shape)
        fb = (bits >> np.uint64(64 - 52)) | np.array(1.0, np.float64).view(np.uint64)
        floats = fb.view(np.float64) - 1.0
    elif dtype == np.float32:
        bits = random_bits32(k, shape)
        fb = (bits >> np.uint32(32 - 23)) | np.array(1.0, np.float32).view(np.uint32)
        floats = fb.view(np.float32) - np.float32(1.0)
    else:
        raise TypeError(dtype)
    minval = dtype.type(minval)
    maxval = dtype.type(maxval)
    return np.maximum(minval, floats * (maxval - minval) + minval)


def normal(k, shape, dtype=np.float64) -> np.ndarray:
    dtype = np.dtype(dtype)
    lo = np.nextafter(dtype.type(-1.0), dtype.type(0.0))
    u = uniform(k, shape, dtype, lo, 1.0)
    return (dtype.type(np.sqrt(2)) * erfinv(u)).astype(dtype)
