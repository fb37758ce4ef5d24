"""GPU adjoint of generate (ggp_generate_vjp_*) against the hand-written FP64 oracle adjoint (itself checked
against finite differences in tests/test_oracle_adjoint.py) and against central finite differences of the GPU
forward pass.

Tolerances: FP64 kernels 1e-8 relative (norm-wise); FP32 kernels 1e-4 for the gradient with respect to xi and
1e-3 for the gradient with respect to the table values (a sum of millions of FP32 terms per bracket).
"""
import numpy as np
import pytest

from oracle import adjoint as oa

from conftest import rel_err
from helpers import as_inputs, oracle_graph, matern32_table, rbf_table

pytestmark = pytest.mark.gpu


def _t(x, dev, dtype=None):
    import torch

    t = torch.as_tensor(np.ascontiguousarray(x), device=dev)
    return t if dtype is None else t.to(dtype)


CASES = [(2000, 2, 100, 10, "rbf", 0.0), (2500, 3, 128, 16, "matern", 0.7), (1500, 2, 64, 20, "rbf", -1.3),
         (1200, 3, 64, 7, "matern", 0.0),
         (3000, 2, 300, 10, "rbf", 0.4)]  # a dense root of five 64-row tiles, the last one ragged


def _table(name):
    return rbf_table(scale=0.3) if name == "rbf" else matern32_table(cutoff=0.4)


@pytest.mark.parametrize("n,d,n0,k,tab,gl", CASES)
def test_vjp_f64_vs_oracle(cuda_device, n, d, n0, k, tab, gl):
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = _table(tab)
    rng = np.random.default_rng(n + k)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)
    rx, rv = oa.generate_vjp(g, (bins, vals), xi, gv, gl)
    gx, gvals = gc.generate_vjp(_t(g.points.astype(np.float64), cuda_device), _t(g.indices, cuda_device),
                                _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device), _t(vals, cuda_device),
                                _t(xi, cuda_device), _t(gv, cuda_device), gl)
    st = gc.last_status()
    assert st["error"] == 0 and st["timeouts"] == 0
    assert rel_err(gx.cpu().numpy(), rx) < 1e-8
    assert rel_err(gvals.cpu().numpy(), rv) < 1e-8


@pytest.mark.parametrize("n,d,n0,k,tab,gl", CASES[:3])
def test_vjp_f32_vs_oracle(cuda_device, n, d, n0, k, tab, gl):
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(_table(tab), np.float32)
    rng = np.random.default_rng(n + k + 1)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)
    rx, rv = oa.generate_vjp(g, (bins, vals), xi, gv, gl)
    f32 = torch.float32
    gx, gvals = gc.generate_vjp(_t(g.points, cuda_device), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device),
                                g.offsets, _t(bins, cuda_device, f32), _t(vals, cuda_device, f32),
                                _t(xi, cuda_device, f32), _t(gv, cuda_device, f32), gl)
    assert rel_err(gx.cpu().numpy(), rx) < 1e-4
    assert rel_err(gvals.cpu().numpy(), rv) < 1e-3


def test_vjp_finite_differences_on_gpu(cuda_device):
    """<grad, direction> equals the central difference of the GPU forward (FP64) along random directions."""
    from graphgp_b200 import graphgp_cuda as gc

    n, d, n0, k = 3000, 2, 128, 12
    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = matern32_table(cutoff=0.4)
    rng = np.random.default_rng(5)
    xi, gv, gl = rng.standard_normal(n), rng.standard_normal(n), 0.5
    args = (_t(g.points.astype(np.float64), cuda_device), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device),
            g.offsets)
    B = _t(bins, cuda_device)
    gx, gvals = gc.generate_vjp(*args, B, _t(vals, cuda_device), _t(xi, cuda_device), _t(gv, cuda_device), gl)
    gx, gvals = gx.cpu().numpy(), gvals.cpu().numpy()

    def loss(x, vv):
        v = gc.generate(*args, B, _t(vv, cuda_device), _t(x, cuda_device)).cpu().numpy()
        ld = float(gc.generate_logdet(args[0], args[2], args[3], B, _t(vv, cuda_device)))
        return float(np.dot(gv, v)) + gl * ld

    h = 1e-6
    for _ in range(4):
        dx = rng.standard_normal(n)
        dv = rng.standard_normal(len(vals)) * 1e-2
        fd = (loss(xi + h * dx, vals + h * dv) - loss(xi - h * dx, vals - h * dv)) / (2 * h)
        an = float(gx @ dx + gvals @ dv)
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(fd))


def test_vjp_differentiation_workload_shape(cuda_device):
    """The differentiation workload's shape at N = 20,000: uniform [0,1]^2, n0 = 256, k = 20, RBF scale 0.1 on
    r = 0 + 1,000 log bins over [1e-5, 1.5], jitter 1e-4, loss 0.5|v - y|^2 + logdet. GPU adjoint (FP64 and
    FP32) against the oracle adjoint."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc
    from oracle import extras as ox
    from oracle import graph as og
    from oracle import refine as orf

    n = 20000
    rng = np.random.default_rng(77)
    pts = rng.uniform(0.0, 1.0, (n, 2)).astype(np.float32)
    g = og.build_graph(pts, n0=256, k=20)
    bins, vals = ox.rbf_kernel(variance=1.0, scale=0.1, r_min=1e-5, r_max=1.5, n_bins=1001, jitter=1e-4)
    y = orf.generate(g, (bins, vals), rng.standard_normal(n)) + 0.01 * rng.standard_normal(n)
    xi = rng.standard_normal(n)
    v = orf.generate(g, (bins, vals), xi)
    refs = {torch.float64: oa.generate_vjp(g, (bins, vals), xi, v - y, 1.0)}
    c32 = as_inputs((bins, vals), np.float32)  # the FP64 oracle on the inputs the FP32 kernels receive
    refs[torch.float32] = oa.generate_vjp(g, c32, xi, orf.generate(g, c32, xi) - y, 1.0)
    args = (_t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets)
    for dt, tol_x, tol_v in ((torch.float64, 1e-8, 1e-8), (torch.float32, 1e-4, 1e-3)):
        rx, rv = refs[dt]
        P = _t(g.points, cuda_device, dt)
        B, V = _t(bins, cuda_device, dt), _t(vals, cuda_device, dt)
        X = _t(xi, cuda_device, dt)
        vg = gc.generate(P, *args, B, V, X)
        gx, gvals = gc.generate_vjp(P, *args, B, V, X, vg - _t(y, cuda_device, dt), 1.0)
        assert gc.last_status()["error"] == 0
        assert rel_err(gx.cpu().numpy(), rx) < tol_x, dt
        assert rel_err(gvals.cpu().numpy(), rv) < tol_v, dt


# shapes outside the four-lane kernel (k > 20, or d not in {2, 3}): the one-thread-per-point adjoint kernel
GENERAL_CASES = [(1500, 2, 64, 24, "rbf", 0.3), (1200, 4, 64, 10, "matern", 0.0), (1000, 3, 64, 32, "matern", -0.4)]


@pytest.mark.parametrize("n,d,n0,k,tab,gl", GENERAL_CASES)
def test_vjp_general_kernel_vs_oracle(cuda_device, n, d, n0, k, tab, gl):
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = _table(tab)
    rng = np.random.default_rng(n + 3 * k)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)
    for dt, tol_x, tol_v in ((torch.float64, 1e-8, 1e-8), (torch.float32, 1e-4, 1e-3)):
        rx, rv = oa.generate_vjp(g, as_inputs((bins, vals), np.float32 if dt == torch.float32 else np.float64), xi,
                                 gv, gl)
        gx, gvals = gc.generate_vjp(_t(g.points, cuda_device, dt), _t(g.indices, cuda_device),
                                    _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device, dt),
                                    _t(vals, cuda_device, dt), _t(xi, cuda_device, dt), _t(gv, cuda_device, dt), gl)
        st = gc.last_status()
        assert st["error"] == 0 and st["timeouts"] == 0, st
        assert rel_err(gx.cpu().numpy(), rx) < tol_x, dt
        assert rel_err(gvals.cpu().numpy(), rv) < tol_v, dt


@pytest.mark.parametrize("n,d,n0,k,tab,gl", [CASES[1], GENERAL_CASES[0]])
def test_vjp_with_forward_values_matches_recompute(cuda_device, n, d, n0, k, tab, gl):
    """Passing generate's output (values=) gives the gradients of the recomputing path: FP64 to 1e-12, FP32 to 1e-6
    (the cotangent scatter adds in a scheduling-dependent order)."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = _table(tab)
    rng = np.random.default_rng(n + 11)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 1e-6)):
        args = (_t(g.points, cuda_device, dt), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                _t(bins, cuda_device, dt), _t(vals, cuda_device, dt), _t(xi, cuda_device, dt))
        v = gc.generate(*args)
        a_x, a_v = gc.generate_vjp(*args, _t(gv, cuda_device, dt), gl)
        b_x, b_v = gc.generate_vjp(*args, _t(gv, cuda_device, dt), gl, values=v)
        assert rel_err(b_x.cpu().numpy(), a_x.cpu().numpy()) < tol, dt
        assert rel_err(b_v.cpu().numpy(), a_v.cpu().numpy()) < tol, dt


# k above the thread-per-point range (10) and up to 20, d in {2, 3}: the forward keeps residuals (13 and 18 pad to
# the 16- and 20-slot kernels)
RESID_CASES = [(2500, 3, 128, 16, "matern", 0.7), (1500, 2, 64, 20, "rbf", -1.3), (1800, 3, 100, 13, "matern", 0.0),
               (2200, 2, 300, 18, "rbf", 0.4)]


@pytest.mark.parametrize("n,d,n0,k,tab,gl", RESID_CASES)
@pytest.mark.parametrize("with_indices", [True, False])
def test_vjp_with_forward_residuals(cuda_device, n, d, n0, k, tab, gl, with_indices):
    """The one-pass forward's residuals (w, a, sigma per refined row) give the gradients of the refactorising
    adjoint: to 1e-5 (FP32; a = K11^-1 v_N is solved in another order) and to the oracle's tolerances."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(_table(tab), np.float32)
    rng = np.random.default_rng(n + 23)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)
    rx, rv = oa.generate_vjp(g, (bins, vals), xi, gv, gl)
    f32 = torch.float32
    idx = _t(g.indices, cuda_device) if with_indices else None
    # without indices every per-point array is in graph order: row r holds original point indices[r]
    xi_t = _t(xi if with_indices else xi[g.indices], cuda_device, f32)
    gv_t = _t(gv if with_indices else gv[g.indices], cuda_device, f32)
    pts_t = _t(g.points, cuda_device, f32)
    args = (pts_t, idx, _t(g.neighbors, cuda_device), g.offsets, _t(bins, cuda_device, f32),
            _t(vals, cuda_device, f32), xi_t)
    v, ld, resid = gc.generate_and_logdet(*args, with_resid=True)
    assert resid is not None and tuple(resid.shape) == (n - n0, 2 * k + 1)
    assert bool(torch.isfinite(resid).all()) and bool((resid[:, 2 * k] > 0).all())
    a_x, a_v = gc.generate_vjp(*args, gv_t, gl, values=v)
    b_x, b_v = gc.generate_vjp(*args, gv_t, gl, values=v, resid=resid)
    st = gc.last_status()
    assert st["error"] == 0 and st["timeouts"] == 0
    assert rel_err(b_x.cpu().numpy(), a_x.cpu().numpy()) < 1e-5
    assert rel_err(b_v.cpu().numpy(), a_v.cpu().numpy()) < 1e-5
    assert rel_err(b_x.cpu().numpy(), rx if with_indices else rx[g.indices]) < 1e-4
    assert rel_err(b_v.cpu().numpy(), rv) < 1e-3


@pytest.mark.parametrize("k", [32, 10])
def test_residuals_absent_outside_four_lane_kernel(cuda_device, k):
    """k = 32 has no four-lane kernel and k = 10 keeps the thread-per-point forward: no residuals (None), and the
    values are those of the call without them."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, d, n0 = 1500, 2, 64
    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = as_inputs(rbf_table(scale=0.3), np.float32)
    f32 = torch.float32
    xi = np.random.default_rng(3).standard_normal(n)
    args = (_t(g.points, cuda_device, f32), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
            _t(bins, cuda_device, f32), _t(vals, cuda_device, f32), _t(xi, cuda_device, f32))
    v, ld, resid = gc.generate_and_logdet(*args, with_resid=True)
    assert resid is None
    v2, ld2 = gc.generate_and_logdet(*args)
    assert torch.equal(v, v2)


@pytest.mark.parametrize("k", [16, 10, 24, 32])
def test_vjp_f32_reconditioned_rows(cuda_device, k):
    """Near-duplicate points (a 2-d shell of radii 10^U(-3, 0)) push some FP32 pivots below tau. The forward
    re-conditions those rows in FP64, and so does the adjoint: w, a and sigma from one FP64 factorisation (the
    four-lane sweep for k <= 20, the warp-per-point sweep for 24 and 32, and the residual-reading sweep, where
    the forward marks the rows). The FP32 gradients stay finite and follow the
    FP64 adjoint; the two FP32 sweeps agree to 1e-5."""
    import torch
    from graphgp_b200 import graphgp_cuda as gc

    n, d, n0 = 20000, 2, 100
    pts, g = oracle_graph(n, d, n0, k, dist="shell")
    bins, vals = as_inputs(rbf_table(scale=0.3), np.float32)
    rng = np.random.default_rng(k)
    xi, gv = rng.standard_normal(n), rng.standard_normal(n)

    def args(dt):
        return (_t(g.points, cuda_device, dt), _t(g.indices, cuda_device), _t(g.neighbors, cuda_device), g.offsets,
                _t(bins, cuda_device, dt), _t(vals, cuda_device, dt), _t(xi, cuda_device, dt))

    a64, a32 = args(torch.float64), args(torch.float32)
    v64 = gc.generate(*a64)
    rx, rv = gc.generate_vjp(*a64, _t(gv, cuda_device, torch.float64), 0.5, values=v64)
    v32 = gc.generate(*a32)
    assert gc.last_status()["fallback_count"] > 0
    ax, av = gc.generate_vjp(*a32, _t(gv, cuda_device, torch.float32), 0.5, values=v32)
    st = gc.last_status()
    assert st["fallback_count"] > 0 and st["error"] == 0
    assert bool(torch.isfinite(ax).all()) and bool(torch.isfinite(av).all())
    # measured on a B200: 1.3e-4 / 3.9e-5 (xi), 2.7e-4 / 2.9e-4 (table) for k = 16 / 10
    assert rel_err(ax.cpu().numpy(), rx.cpu().numpy()) < 2e-3
    assert rel_err(av.cpu().numpy(), rv.cpu().numpy()) < 2e-3
    v2, ld, resid = gc.generate_and_logdet(*a32, with_resid=True)
    if resid is not None:
        assert bool((resid[:, 2 * k] < 0).any())
        bx, bv = gc.generate_vjp(*a32, _t(gv, cuda_device, torch.float32), 0.5, values=v2, resid=resid)
        assert rel_err(bx.cpu().numpy(), ax.cpu().numpy()) < 1e-5
        assert rel_err(bv.cpu().numpy(), av.cpu().numpy()) < 1e-5
