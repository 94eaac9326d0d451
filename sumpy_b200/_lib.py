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

CU_SOURCES = ["capi.cu", "p2p.cu", "expansions.cu", "m2l.cu", "m2l_tc.cu", "helmholtz.cu",
              "helmholtz_items.cu", "helmholtz_l2p.cu", "p2p_matrix.cu", "laplace_items_f64.cu",
              "tree_gpu.cu", "qbx.cu"]

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


OBJ_DIR = ROOT / "_build"


def build_cuda_library(force=False, extra_flags=()) -> Path:
    """Compile each CUDA source to an object under ``_build/`` (in parallel,
    only those older than their source or a header), then link the shared
    library."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = _cuda_sources()
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    newest_header = max(p.stat().st_mtime for p in headers)
    objs = [OBJ_DIR / (s.stem + ".o") for s in srcs]
    # without objects (a copied tree): a library newer than every source is current
    if not force and not extra_flags and not any(o.exists() for o in objs) and \
            CUDA_LIB.exists() and CUDA_LIB.stat().st_mtime >= max(
                newest_header, max(p.stat().st_mtime for p in srcs)):
        return CUDA_LIB
    OBJ_DIR.mkdir(exist_ok=True)
    stale = [(s, o) for s, o in zip(srcs, objs)
             if force or extra_flags or not o.exists()
             or o.stat().st_mtime < max(s.stat().st_mtime, newest_header)]

    def compile_one(so):
        s, o = so
        _run([NVCC, *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-c",
              "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "-I", str(INCLUDE),
              "-o", str(o), str(s), *extra_flags])

    if stale:
        with ThreadPoolExecutor(max_workers=len(stale)) as ex:
            list(ex.map(compile_one, stale))
    if stale or not CUDA_LIB.exists() or \
            CUDA_LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        _run([NVCC, *ARCH_FLAGS, "-shared", "-ccbin", HOST_CXX, "-o", str(CUDA_LIB),
              *map(str, objs)])
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
