"""CPU-side checks of the C-ABI library: it loads, and it exports every entry point include/graphgp_b200.h
declares (no compute calls; those need a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "graphgp_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|uint64_t|void|double|const char\*)\s+(ggp_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for base in ("build_tree", "query_preceding_neighbors", "query_neighbors", "compute_depths", "order_by_depth",
                 "build_graph", "refine", "refine_inv", "refine_logdet"):
        assert any(s.startswith("ggp_" + base) for s in syms), base


def test_library_loads_and_exports_all_symbols():
    from graphgp_b200 import _lib

    path = _lib.lib_path()
    if not path.exists():
        pytest.fail(f"library not built: {path}")
    lib = ctypes.CDLL(str(path))  # resolves every undefined symbol (RTLD_NOW below)
    lib = ctypes.CDLL(str(path), mode=ctypes.RTLD_GLOBAL | 2)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.exported_symbols()) == set(declared_symbols())


def test_version_and_workspace_size_without_gpu():
    from graphgp_b200 import _lib

    lib = _lib.load()
    assert lib.ggp_version().startswith(b"graphgp_b200")
    sz = lib.ggp_workspace_size(_lib.OPS["GENERATE"], 1 << 20, 3, 1024, 16, 2049, 100, 4)
    assert sz >= (1 << 20) * 4 + 1024 * 1024 * 8


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from graphgp_b200 import _lib

    monkeypatch.setattr(_lib, "_LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.load()


def test_dataflow_width_knob():
    """ggp_set_dataflow_width / ggp_get_dataflow_width are host-only (no device needed): negative widths clamp to
    0 (one full persistent grid), and the default is restored afterwards."""
    from graphgp_b200 import _lib

    lib = _lib.load()
    old = lib.ggp_get_dataflow_width()
    try:
        lib.ggp_set_dataflow_width(8.0)
        assert lib.ggp_get_dataflow_width() == 8.0
        lib.ggp_set_dataflow_width(-3.0)
        assert lib.ggp_get_dataflow_width() == 0.0
    finally:
        lib.ggp_set_dataflow_width(old)
    assert lib.ggp_get_dataflow_width() == old == 4.0


def _header_params():
    """{name: (return kind, [parameter kinds])} from the header's declarations, comments removed. Kinds: 'P'
    (any pointer, the stream handle included), 'I' (int / int32_t / enum), 'I64', 'U64' (uint64_t, size_t),
    'D' (double), 'V' (void)."""
    text = re.sub(r"/\*.*?\*/", " ", HEADER.read_text(), flags=re.S)
    decls = re.findall(r"^\s*((?:const\s+)?\w+\s*\*?)\s+(ggp_\w+)\s*\(([^;{]*?)\)\s*;", text, re.M | re.S)

    def kind(decl):
        decl = " ".join(decl.split())
        if "*" in decl or decl.startswith("ggp_stream_t"):
            return "P"
        base = decl.replace("const ", "").split()[0]
        return {"int": "I", "int32_t": "I", "int64_t": "I64", "uint64_t": "U64", "size_t": "U64", "double": "D",
                "void": "V", "float": "F"}[base]

    out = {}
    for ret, name, params in decls:
        ps = [p for p in (s.strip() for s in params.split(",")) if p and p != "void"]
        out[name] = (kind(ret), [kind(p) for p in ps])
    return out


def _ctypes_kind(t):
    if t is None:
        return "V"
    if t in (ctypes.c_void_p, ctypes.c_char_p) or hasattr(t, "_type_") and isinstance(t._type_, type):
        return "P"
    return {ctypes.c_int: "I", ctypes.c_int64: "I64", ctypes.c_uint64: "U64", ctypes.c_size_t: "U64",
            ctypes.c_double: "D", ctypes.c_float: "F"}[t]


def test_ctypes_signatures_match_header():
    """Every ctypes signature in graphgp_b200/_lib.py has the header's parameter count and kinds, in order (an
    argument added on one side only would otherwise shift every later argument)."""
    from graphgp_b200 import _lib

    hdr = _header_params()
    assert set(hdr) == set(declared_symbols())
    for name, (args, res) in _lib._SIGS.items():
        h_ret, h_args = hdr[name]
        got = [_ctypes_kind(a) for a in args]
        assert got == h_args, (name, got, h_args)
        assert _ctypes_kind(res) == h_ret, (name, res, h_ret)
