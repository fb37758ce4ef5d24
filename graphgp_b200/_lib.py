"""ctypes binding of the in-tree CUDA library ``libgraphgp_b200.so`` (C ABI declared in include/graphgp_b200.h).

There is no CPU fallback: importing the functions that need the library raises if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libgraphgp_b200.so"

GGP_OK = 0
GGP_ERR_INVALID = 1
GGP_ERR_CUDA = 2
GGP_ERR_TIMEOUT = 3
GGP_ERR_UNSUPPORTED = 4
GGP_ERR_WORKSPACE = 5

OPS = dict(
    BUILD_TREE=1, QUERY_NEIGHBORS=2, BUILD_GRAPH=3, COMPUTE_DEPTHS=4, ORDER_BY_DEPTH=5, REFINE=6, REFINE_INV=7,
    REFINE_LOGDET=8, GENERATE=9, GENERATE_INV=10, GENERATE_LOGDET=11, DENSE=12, GENERATE_VJP=13,
)


class GraphGPError(RuntimeError):
    """A non-zero status from the CUDA library."""

    def __init__(self, code: int, where: str):
        names = {1: "invalid argument", 2: "CUDA error", 3: "device wait timed out", 4: "unsupported size",
                 5: "workspace too small"}
        super().__init__(f"{where}: {names.get(code, 'error')} (code {code})")
        self.code = code


class GraphGPValueError(GraphGPError, ValueError):
    pass


def check(code: int, where: str) -> None:
    if code == GGP_OK:
        return
    if code == GGP_ERR_INVALID:
        raise GraphGPValueError(code, where)
    raise GraphGPError(code, where)


class Status(C.Structure):
    _fields_ = [("error", C.c_uint32), ("nan_seen", C.c_uint32), ("fallback_count", C.c_uint32),
                ("timeouts", C.c_uint32)]


_P = C.c_void_p
_I64 = C.c_int64
_I = C.c_int
_D = C.c_double
_U64 = C.c_uint64
_SZ = C.c_size_t

# (name, argtypes) for every entry point; the suffix-less tuple lists the f32 variant's types, and the
# f64 variant differs only in pointer element type (all pointers are void* here) and the missing tau.
_SIGS = {
    "ggp_version": ([], C.c_char_p),
    "ggp_workspace_size": ([_I, _I64, _I, _I64, _I, _I, _I, _I], _SZ),
    "ggp_launch_count": ([], C.c_uint64),
    "ggp_set_dataflow_width": ([C.c_double], None),
    "ggp_get_dataflow_width": ([], C.c_double),
    "ggp_read_status": ([_P, C.POINTER(Status), _P], _I),
    "ggp_build_tree_f32": ([_P, _I64, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_build_tree_f64": ([_P, _I64, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_query_preceding_neighbors_f32": ([_P, _P, _I64, _I, _I64, _I, _P, _P, _SZ, _P], _I),
    "ggp_query_preceding_neighbors_f64": ([_P, _P, _I64, _I, _I64, _I, _P, _P, _SZ, _P], _I),
    "ggp_query_neighbors_f32": ([_P, _P, _I64, _I, _P, _P, _I64, _I, _P, _P, _SZ, _P], _I),
    "ggp_query_neighbors_f64": ([_P, _P, _I64, _I, _P, _P, _I64, _I, _P, _P, _SZ, _P], _I),
    "ggp_compute_depths": ([_P, _I64, _I64, _I, _P, _P, _SZ, _P], _I),
    "ggp_order_by_depth_f32": ([_P, _P, _P, _P, _I64, _I, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_order_by_depth_f64": ([_P, _P, _P, _P, _I64, _I, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_build_graph_f32": ([_P, _I64, _I, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_build_graph_f64": ([_P, _I64, _I, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_refine_f32": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _D, _U64, _P, _SZ, _P], _I),
    "ggp_refine_f64": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _U64, _P, _SZ, _P], _I),
    "ggp_refine_inv_f32": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _D, _P, _SZ, _P], _I),
    "ggp_refine_inv_f64": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_refine_logdet_f32": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _D, _P, _SZ, _P], _I),
    "ggp_refine_logdet_f64": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _SZ, _P], _I),
    "ggp_refine_logdet_f32_noalloc": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _D, _P], _I),
    "ggp_dense_f32": ([_I, _P, _I64, _I, _P, _P, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_dense_f64": ([_I, _P, _I64, _I, _P, _P, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_generate_f32": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _D, _U64, _P, _SZ, _P], _I),
    "ggp_generate_f64": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _U64, _P, _SZ, _P], _I),
    "ggp_generate_inv_f32": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _D, _P, _SZ, _P], _I),
    "ggp_generate_inv_f64": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _SZ, _P], _I),
    "ggp_generate_logdet_f32": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _D, _P, _SZ, _P], _I),
    "ggp_generate_logdet_f64": ([_P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _SZ, _P], _I),
    "ggp_generate_vjp_f32": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _D, _P, _P, _D, _P,
                              _SZ, _P], _I),
    "ggp_generate_vjp_f64": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _D, _P, _P, _P, _SZ,
                              _P], _I),
    "ggp_wait_probe": ([_U64, C.POINTER(C.c_int), _P, _SZ, _P], _I),
    "ggp_fma_probe": ([_I, _I, _I, C.POINTER(C.c_double), _P, _SZ, _P], _I),
    "ggp_generate_and_logdet_f32": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _P, _D, _U64,
                                     _P, _SZ, _P], _I),
    "ggp_generate_vjp_resid_f32": ([_P, _P, _I64, _I, _I64, _P, _I, _P, _I, _P, _P, _I, _P, _P, _P, _P, _D, _P, _P, _D,
                                    _P, _SZ, _P], _I),
    "ggp_request_buffer_size": ([_I, _I64, _I, _I64, _I, _I, _I], _SZ),
    "ggp_request_f32": ([_I, _P, _I64, _I, _I64, _I, _P, _P, _I, _P, _P, _P, _D, _P, _SZ, _P], _I),
    "ggp_request_f64": ([_I, _P, _I64, _I, _I64, _I, _P, _P, _I, _P, _P, _P, _P, _SZ, _P], _I),
    "ggp_request_host_sizes": ([_I, _I64, _I, _I64, _I, _I, _I, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)], _I),
    "ggp_request_host_f32": ([_I, _P, _I64, _I, _I64, _I, _P, _P, _I, _P, _P, _P, C.POINTER(Status), _D, _P, _SZ,
                              _P, _SZ, _P], _I),
    "ggp_request_host_f64": ([_I, _P, _I64, _I, _I64, _I, _P, _P, _I, _P, _P, _P, C.POINTER(Status), _P, _SZ, _P,
                              _SZ, _P], _I),
}

_lib = None


def lib_path() -> Path:
    return _LIB_PATH


def load():
    """Load the library (raising ImportError if it has not been built) and bind every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"graphgp_b200 CUDA library not built: {_LIB_PATH} is missing "
                          "(run `python -m graphgp_b200.build`)")
    lib = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGS)
