"""The small plain-method configuration run exactly, on the GPU, against the FP64 oracle.

N = 100,000 points in d = 2, standard normal float32 from NumPy seed 99, xi standard normal from the same
generator; build_graph(n0 = 100, k = 10); RBF kernel variance 1, scale 0.3, tabulated at r = 0 plus 1,000
log-spaced bins on [1e-4, 10] (1,001 entries), jitter 1e-4. The graph must match the oracle bit for bit; FP32
generate, inverse and log-determinant must be within 1e-4 relative error of the FP64 oracle on the same inputs
(the table rounded to FP32, as the FP32 kernels receive it; reference graphgp/refine.py:21-56, 162-183,
234-240), and the FP64 kernels within 1e-9.
"""
import numpy as np
import pytest

from conftest import rel_err
from oracle import extras as ox
from oracle import graph as og
from oracle import refine as orf

from helpers import as_inputs

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL64 = 1e-9


def _t(x, dev, dtype=None):
    import torch

    t = torch.as_tensor(np.ascontiguousarray(x), device=dev)
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def config1():
    rng = np.random.default_rng(99)
    pts = rng.standard_normal((100_000, 2)).astype(np.float32)
    xi = rng.standard_normal(100_000)
    g = og.build_graph(pts, n0=100, k=10)
    bins, vals = ox.rbf_kernel(variance=1.0, scale=0.3, r_min=1e-4, r_max=10.0, n_bins=1001, jitter=1e-4)
    refs = {}
    for dtype in ("float32", "float64"):  # the FP64 oracle on the inputs each kernel receives
        cov = as_inputs((bins, vals), getattr(np, dtype))
        ref = orf.generate(g, cov, xi)
        refs[dtype] = (ref, orf.generate_inv(g, cov, ref.astype(np.float32)), orf.generate_logdet(g, cov))
    return pts, xi, g, (bins, vals), refs


def test_config1_graph_bit_exact(cuda_device, config1):
    from graphgp_b200 import graphgp_cuda as gc

    pts, _, g, _, _ = config1
    gp, gi, gn, gd, offs = gc.build_graph(_t(pts, cuda_device), n0=100, k=10, return_offsets=True)
    assert list(offs) == list(g.offsets)
    assert np.array_equal(gi.cpu().numpy(), g.indices)
    assert np.array_equal(gn.cpu().numpy(), g.neighbors)
    assert np.array_equal(gp.cpu().numpy(), g.points)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_config1_values_inverse_logdet(cuda_device, config1, dtype):
    import torch

    from graphgp_b200 import graphgp_cuda as gc

    pts, xi, g, (bins, vals), refs = config1
    ref, ref_inv, ref_ld = refs[dtype]
    tdt = getattr(torch, dtype)
    tol = TOL32 if dtype == "float32" else TOL64
    P = _t(g.points, cuda_device, tdt)
    I, NB = _t(g.indices, cuda_device), _t(g.neighbors, cuda_device)
    B, V = _t(bins, cuda_device, tdt), _t(vals, cuda_device, tdt)
    out = gc.generate(P, I, NB, g.offsets, B, V, _t(xi, cuda_device, tdt))
    assert gc.last_status()["error"] == 0
    assert rel_err(out.cpu().numpy(), ref) < tol
    # the inverse of the FP32-rounded oracle values (the oracle inverts the same rounded values)
    back = gc.generate_inv(P, I, NB, g.offsets, B, V, _t(ref.astype(np.float32), cuda_device, tdt))
    st = gc.last_status()
    assert st["error"] == 0 and st["nan_seen"] == 0
    assert rel_err(back.cpu().numpy(), ref_inv) < tol
    ld = float(gc.generate_logdet(P, NB, g.offsets, B, V))
    assert abs(ld - ref_ld) <= tol * abs(ref_ld)
