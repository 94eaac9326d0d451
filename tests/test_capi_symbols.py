"""The C-ABI library exports every function the headers declare; the
ctypes declarations cover them all (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import pytest

from sumpy_b200 import _capi, _lib

ROOT = Path(__file__).resolve().parents[1]


def declared(header):
    txt = (ROOT / "include" / header).read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sumpy_\w+)\s*\(", txt)))


def test_cuda_library_exports_header_symbols():
    path = _lib.build_cuda_library()
    lib = ctypes.CDLL(str(path))
    names = declared("sumpy_b200.h")
    assert names, "no declarations found"
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    assert sorted(_capi.exported_names()) == names


def test_tree_library_exports_header_symbols():
    lib = _lib.load_tree_library()
    for n in declared("sumpy_b200_tree.h"):
        assert hasattr(lib, n), f"missing export {n}"


def test_no_gpu_call_raises_cleanly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = ctypes.CDLL(str(_lib.build_cuda_library()))
    lib.sumpy_version.restype = ctypes.c_int
    assert lib.sumpy_version() >= 1
