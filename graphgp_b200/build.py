"""Build the in-tree CUDA library ``graphgp_b200/libgraphgp_b200.so`` for sm_100a.

Every ``csrc/*.cu`` and ``csrc/inst/*.cu`` unit is compiled with nvcc in parallel (the register-resident
kernel instantiations are split across units for that reason) and linked with ``-shared``. A unit is
rebuilt when it, or any header it includes (transitively), is newer than its object file.

Usage: ``python -m graphgp_b200.build [--force] [--jobs N] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgraphgp_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-diag-suppress", "1886", f"-I{ROOT / 'include'}"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the graphgp_b200 CUDA library cannot be built")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted((CSRC / "inst").glob("*.cu"))


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps_mtime(src: Path, seen=None) -> float:
    """Newest modification time of `src` and every quoted header it includes, transitively."""
    seen = set() if seen is None else seen
    if src in seen or not src.exists():
        return 0.0
    seen.add(src)
    t = src.stat().st_mtime
    for inc in _INCLUDE.findall(src.read_text()):
        t = max(t, _deps_mtime((src.parent / inc).resolve(), seen))
    return t


def _obj_for(src: Path) -> Path:
    rel = src.relative_to(CSRC)
    return BUILD / (str(rel).replace(os.sep, "__") + ".o")


def _compile(src: Path, verbose: bool) -> tuple[Path, str]:
    obj = _obj_for(src)
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stdout + res.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    todo = []
    for s in srcs:
        o = _obj_for(s)
        if force or not o.exists() or o.stat().st_mtime < _deps_mtime(s.resolve()):
            todo.append(s)
    logs = []
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
                logs.append((obj, log))
    objs = [_obj_for(s) for s in srcs]
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        for obj, log in logs:
            sys.stdout.write(f"==== {obj.name}\n{log}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
