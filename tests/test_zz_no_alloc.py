"""The log-determinant entry point that allocates nothing (ggp_refine_logdet_f32_noalloc).

Callers that cannot allocate device memory -- a framework holding nearly all of the GPU in its own pool, a
foreign-function handler without a scratch allocator, a loop that must not enter an allocator -- use this
variant, which takes its scratch from a fixed array inside the library instead of a caller workspace. These
tests call it through the C ABI and check it against ggp_refine_logdet_f32 (same kernel, caller workspace)
on two calls in a row, so that whatever the first call leaves in the shared array cannot leak into the
second; and that inputs beyond the array's limit are refused. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import as_inputs, oracle_graph, matern32_table
from oracle import refine as orf

pytestmark = pytest.mark.gpu

TOL32 = 1e-4


def _t(x, dev, dtype=None):
    import torch

    t = torch.as_tensor(np.ascontiguousarray(x), device=dev)
    return t if dtype is None else t.to(dtype)


def _logdet_with_workspace(lib, args, dev):
    import torch

    (P, n, d, n0, NB, k, OF, nofs, B, V, nb) = args
    size = lib.ggp_workspace_size(8, n, d, n0, k, nb, nofs, 4)  # GGP_OP_REFINE_LOGDET
    ws = torch.empty(size, dtype=torch.uint8, device=dev)
    out = torch.empty((), dtype=torch.float64, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.ggp_refine_logdet_f32(C.c_void_p(P.data_ptr()), n, d, n0, C.c_void_p(NB.data_ptr()), k,
                                   C.c_void_p(OF.data_ptr()), nofs, C.c_void_p(B.data_ptr()),
                                   C.c_void_p(V.data_ptr()), nb, C.c_void_p(out.data_ptr()), 1e-5,
                                   C.c_void_p(ws.data_ptr()), size, s)
    assert rc == 0
    return float(out)


def _logdet_noalloc(lib, args, dev):
    import torch

    (P, n, d, n0, NB, k, OF, nofs, B, V, nb) = args
    out = torch.full((), float("nan"), dtype=torch.float64, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.ggp_refine_logdet_f32_noalloc(C.c_void_p(P.data_ptr()), n, d, n0, C.c_void_p(NB.data_ptr()), k,
                                           C.c_void_p(OF.data_ptr()), nofs, C.c_void_p(B.data_ptr()),
                                           C.c_void_p(V.data_ptr()), nb, C.c_void_p(out.data_ptr()), 1e-5, s)
    assert rc == 0
    return float(out)


def _inputs(dev, n, d, n0, k):
    import torch

    pts, g = oracle_graph(n, d, n0, k)
    bins, vals = matern32_table(cutoff=0.5)
    f32 = torch.float32
    args = (_t(g.points, dev), n, d, n0, _t(g.neighbors.astype(np.int32), dev), k,
            _t(np.asarray(g.offsets, np.int32), dev), len(g.offsets), _t(bins, dev, f32), _t(vals, dev, f32),
            len(bins))
    return args, g, (bins, vals)


@pytest.mark.parametrize("n,d,n0,k", [(3000, 3, 256, 16), (2500, 2, 100, 10)])
def test_noalloc_logdet_matches_workspace_version_twice(cuda_device, n, d, n0, k):
    from graphgp_b200 import _lib

    lib = _lib.load()
    args, g, cov = _inputs(cuda_device, n, d, n0, k)
    ref = _logdet_with_workspace(lib, args, cuda_device)
    first = _logdet_noalloc(lib, args, cuda_device)
    second = _logdet_noalloc(lib, args, cuda_device)
    for got in (first, second):
        assert abs(got - ref) <= TOL32 * abs(ref)
    oracle = orf.refine_logdet(g.points, g.neighbors, g.offsets, as_inputs(cov, np.float32))
    assert abs(second - oracle) <= TOL32 * abs(oracle)


def _call_noalloc(lib, dev, P, n, d, n0, NB, k, OF, nofs, B, V, nb):
    import torch

    out = torch.full((), float("nan"), dtype=torch.float64, device=dev)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.ggp_refine_logdet_f32_noalloc(C.c_void_p(P.data_ptr()), n, d, n0, C.c_void_p(NB.data_ptr()), k,
                                           C.c_void_p(OF.data_ptr()), nofs, C.c_void_p(B.data_ptr()),
                                           C.c_void_p(V.data_ptr()), nb, C.c_void_p(out.data_ptr()), 1e-5, s)
    return rc, out


def test_noalloc_limits_at_the_boundary(cuda_device):
    """The two stated limits, each on its own: 4097 table entries together with 100,000 offsets is accepted and
    gives the same log-determinant as the workspace version; 100,001 offsets or 4098 table entries is refused
    before anything runs. The offsets are the graph's own, padded with empty batches at the end (allowed: a
    batch may be empty, and the log-determinant waits on nothing)."""
    import torch

    from graphgp_b200 import _lib

    lib = _lib.load()
    pts, g = oracle_graph(3000, 3, 256, 16)
    P = _t(g.points, cuda_device)
    NB = _t(g.neighbors.astype(np.int32), cuda_device)
    f32 = torch.float32

    def table(nb):
        bins, vals = matern32_table(cutoff=0.5, n_bins=nb)
        return _t(bins, cuda_device, f32), _t(vals, cuda_device, f32)

    def padded(count):
        offs = np.asarray(g.offsets, np.int32)
        return _t(np.concatenate([offs, np.full(count - len(offs), offs[-1], np.int32)]), cuda_device)

    B, V = table(4097)
    OF = padded(100000)
    args = (P, 3000, 3, 256, NB, 16, _t(np.asarray(g.offsets, np.int32), cuda_device), len(g.offsets), B, V, 4097)
    ref = _logdet_with_workspace(lib, args, cuda_device)
    rc, out = _call_noalloc(lib, cuda_device, P, 3000, 3, 256, NB, 16, OF, 100000, B, V, 4097)
    assert rc == 0
    assert abs(float(out) - ref) <= TOL32 * abs(ref)

    OF1 = padded(100001)
    rc, out = _call_noalloc(lib, cuda_device, P, 3000, 3, 256, NB, 16, OF1, 100001, B, V, 4097)
    assert rc == _lib.GGP_ERR_UNSUPPORTED
    B2, V2 = table(4098)
    rc, out = _call_noalloc(lib, cuda_device, P, 3000, 3, 256, NB, 16, OF, 100000, B2, V2, 4098)
    assert rc == _lib.GGP_ERR_UNSUPPORTED
    rc, out = _call_noalloc(lib, cuda_device, P, 3000, 3, 256, NB, 16, OF, 400000, B, V, 4097)
    assert rc == _lib.GGP_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert torch.isnan(out).item()  # refused calls write nothing
