"""Build and load the native libraries of sumpy_b200.

* ``libsumpy_b200.so`` -- the sm_100a CUDA kernels behind the C-ABI declared
  in ``include/sumpy_b200.h`` (sources ``sumpy_b200/csrc/*.cu``).
* ``libsumpy_b200_tree.so`` -- the host octree / interaction-list builder
  declared in ``include/sumpy_b200_tree.h`` (source ``sumpy_b200/csrc/tree.cpp``).

Both are built in-tree (next to this file). Nothing here falls back to a
Python or CPU implementation of the FMM stages: if the CUDA library is
missing or fails to load, :func:`load_cuda_library` raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
CUDA_LIB = PKG / "libsumpy_b200.so"
TREE_LIB = PKG / "libsumpy_b200_tree.so"

NVCC = os.environ.get("SUMPY_B200_NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = os.environ.get("SUMPY_B200_HOST_CXX", "/usr/bin/g++")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["capi.cu", "p2p.cu", "expansions.cu", "m2l.cu", "m2l_tc.cu", "helmholtz.cu"]

_lock = threading.Lock()
_cuda = None
_tree = None


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return res


def build_tree_library(force=False) -> Path:
    src = CSRC / "tree.cpp"
    if force or not TREE_LIB.exists() or TREE_LIB.stat().st_mtime < src.stat().st_mtime:
        _run([HOST_CXX, "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
              "-I", str(INCLUDE), "-o", str(TREE_LIB), str(src)])
    return TREE_LIB


def _cuda_sources():
    return [CSRC / s for s in CU_SOURCES]


def build_cuda_library(force=False, extra_flags=()) -> Path:
    srcs = _cuda_sources()
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest = max(p.stat().st_mtime for p in srcs + headers)
    if force or not CUDA_LIB.exists() or CUDA_LIB.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared",
               "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "-I", str(INCLUDE),
               "-o", str(CUDA_LIB), *map(str, srcs), *extra_flags]
        _run(cmd)
    return CUDA_LIB


def load_tree_library():
    global _tree
    with _lock:
        if _tree is None:
            if not TREE_LIB.exists():
                build_tree_library()
            lib = ctypes.CDLL(str(TREE_LIB))
            lib.sumpy_tree_last_error.restype = ctypes.c_char_p
            _tree = lib
    return _tree


def load_cuda_library():
    """Load ``libsumpy_b200.so``; raise if it is absent (no fallback)."""
    global _cuda
    with _lock:
        if _cuda is None:
            if not CUDA_LIB.exists():
                raise RuntimeError(
                    f"{CUDA_LIB} is missing: build it with "
                    "`python -c 'import sumpy_b200._lib as l; l.build_cuda_library()'` "
                    "(sumpy_b200 has no CPU fallback)")
            lib = ctypes.CDLL(str(CUDA_LIB))
            from sumpy_b200 import _capi
            _capi.declare(lib)
            _cuda = lib
    return _cuda
