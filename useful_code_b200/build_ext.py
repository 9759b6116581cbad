"""Build the in-tree CUDA library ``liblmm_b200.so`` for sm_100a.

Every ``csrc/*.cu`` file is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into ``_build/``
and linked into ``useful_code_b200/liblmm_b200.so``.  Objects are rebuilt
only when a source or header is newer than the object.  Run directly
(``python -m useful_code_b200.build_ext``) or through ``__graft_entry__.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "lmm_b200"
LIB = PKG / "liblmm_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "-I" + str(ROOT / "include"),
]


def nvcc() -> str:
    exe = shutil.which("nvcc")
    if exe:
        return exe
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))


CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I" + str(ROOT / "include")]


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.stem + (".cpp.o" if src.suffix == ".cpp" else ".o"))
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    if src.suffix == ".cpp":
        cmd = [shutil.which("g++") or "g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = list(extra or [])
    BUILD.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), sources))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
