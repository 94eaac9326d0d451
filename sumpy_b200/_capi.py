"""ctypes declarations of the C-ABI in ``include/sumpy_b200.h``.

Every exported entry point is declared here with its exact argument types;
:func:`call` checks the returned status and raises ``RuntimeError`` with the
library's message, mirroring how sumpy surfaces kernel failures as Python
exceptions.
"""
from __future__ import annotations

import ctypes

i32 = ctypes.c_int32
i64 = ctypes.c_int64
cint = ctypes.c_int
dbl = ctypes.c_double
ptr = ctypes.c_void_p

# name -> argument types (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "sumpy_version": [],
    "sumpy_last_error": [],
    "sumpy_p2p_from_csr_f64": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64, ptr,
                               ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_p2p_from_csr_mixed": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64, ptr,
                                 ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_p2p_direct_f64": [i64, ptr, i64, i64, ptr, i64, ptr, ptr, dbl, ptr, ptr],
    "sumpy_p2p_direct_grad_f64": [i64, ptr, i64, i64, ptr, i64, ptr, ptr, dbl, ptr, ptr, ptr],
    "sumpy_p2p_from_csr_grad_f64": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64, ptr,
                                    ptr, i64, ptr, dbl, ptr, ptr, ptr],
    "sumpy_p2p_from_csr_grad_mixed": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64, ptr,
                                      ptr, i64, ptr, dbl, ptr, ptr, ptr],
    "sumpy_e2p_from_single_box_grad_f64": [cint, dbl, i32, ptr, ptr, i64, i32, ptr, ptr, ptr,
                                           ptr, i64, dbl, ptr, ptr, ptr],
    "sumpy_e2p_from_csr_grad_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, i32, ptr, ptr,
                                    ptr, ptr, i64, dbl, ptr, ptr, ptr],
    "sumpy_p2e_from_single_box_f64": [cint, dbl, i32, ptr, ptr, i64, ptr, ptr, ptr, i64,
                                      ptr, i32, ptr, ptr],
    "sumpy_p2e_from_csr_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, ptr,
                               i64, ptr, i32, ptr, ptr],
    "sumpy_e2e_from_children_f64": [cint, cint, dbl, dbl, i32, ptr, ptr, i64, ptr, i64,
                                    i32, ptr, i32, ptr, ptr],
    "sumpy_e2e_from_parent_f64": [cint, cint, dbl, dbl, i32, ptr, ptr, ptr, i64, i32, ptr,
                                  i32, ptr, ptr],
    "sumpy_m2l_translation_classes_f64": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr,
                                          i32, ptr, i32, ptr, i32, ptr, ptr],
    "sumpy_split_tf32x2": [i64, i32, i32, ptr, i32, i32, ptr, ptr, ptr],
    "sumpy_split_f16x2_rowscale": [i64, i32, i32, ptr, i32, i32, ptr, ptr, ptr, ptr],
    "sumpy_m2l_translation_classes_f16x3": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr,
                                            i32, ptr, ptr, ptr, i32, i32, i32, i32, ptr, ptr,
                                            ptr, i32, ptr, ptr, ptr],
    "sumpy_helmholtz_m2l_translation_classes_f16x3": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                                      ptr, ptr, i32, ptr, ptr, ptr, i32, i32,
                                                      i32, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                                      ptr],
    "sumpy_class_gemm_f16x3": [i32, i32, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr, i32, ptr,
                               ptr, ptr, i32, i32, i32, i32, ptr, ptr, ptr, i32, ptr, ptr,
                               ptr],
    "sumpy_set_tc_wait_cycles": [i64],
    "sumpy_tree_gpu_build": [i64, ptr, ptr, ptr, i64, ptr, ptr, ptr, i32, ptr, ptr, cint, cint,
                             ptr, dbl, ptr, ptr],
    "sumpy_tree_gpu_array_info": [ptr, ctypes.c_char_p, ptr, ptr],
    "sumpy_tree_gpu_array_copy": [ptr, ctypes.c_char_p, ptr, i64, cint, ptr],
    "sumpy_tree_gpu_free": [ptr],
    # QBX layer potentials (order, mode, axis[, k], ...)
    "sumpy_qbx_lpot_laplace_f64": [cint, cint, cint, i64, ptr, i64, ptr, i64, i64, ptr, i64,
                                   ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_qbx_lpot_helmholtz_f64": [cint, cint, cint, dbl, i64, ptr, i64, ptr, i64, i64, ptr,
                                     i64, ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_qbx_matrix_laplace_f64": [cint, cint, cint, i64, ptr, i64, ptr, i64, i64, ptr, i64,
                                     ptr, i64, dbl, ptr, ptr],
    "sumpy_qbx_matrix_helmholtz_f64": [cint, cint, cint, dbl, i64, ptr, i64, ptr, i64, i64,
                                       ptr, i64, ptr, i64, dbl, ptr, ptr],
    "sumpy_qbx_matrix_subset_laplace_f64": [cint, cint, cint, i64, ptr, ptr, ptr, i64, ptr,
                                            i64, ptr, i64, ptr, i64, dbl, ptr, ptr],
    "sumpy_qbx_matrix_subset_helmholtz_f64": [cint, cint, cint, dbl, i64, ptr, ptr, ptr, i64,
                                              ptr, i64, ptr, i64, ptr, i64, dbl, ptr, ptr],
    "sumpy_get_tc_wait_cycles": [],
    "sumpy_m2l_translation_classes_tf32x3": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr,
                                             i32, ptr, ptr, i32, i32, i32, i32, ptr, ptr, i32,
                                             ptr, ptr, ptr],
    "sumpy_m2l_translation_classes_tf32x3_noalloc": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                                     ptr, ptr, i32, ptr, ptr, i32, i32, i32,
                                                     i32, ptr, i32, ptr, ptr, ptr],
    "sumpy_e2p_from_single_box_f64": [cint, dbl, i32, ptr, ptr, i64, i32, ptr, ptr, ptr,
                                      ptr, i64, dbl, ptr, ptr],
    "sumpy_e2p_from_csr_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, i32, ptr, ptr, ptr,
                               ptr, i64, dbl, ptr, ptr],
    "sumpy_e2p_from_csr_mixed": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, i32, ptr, ptr, ptr,
                                 ptr, i64, dbl, ptr, ptr],
    "sumpy_p2e_from_csr_mixed": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, ptr,
                                 i64, ptr, i32, ptr, ptr],
    "sumpy_p2e_from_single_box_levels_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr,
                                             ptr, i64, ptr, ptr, ptr],
    "sumpy_e2p_from_single_box_packed_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr,
                                             i64, dbl, ptr, ptr],
    "sumpy_mpoles_to_f32": [cint, i64, ptr, ptr, ptr],
    "sumpy_p2p_matrix_f64": [i64, ptr, i64, i64, ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_helmholtz_e2p_from_single_box_packed_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64,
                                                       ptr, ptr, i64, dbl, ptr, ptr],
    "sumpy_helmholtz_p2p_matrix_f64": [i64, ptr, i64, i64, ptr, i64, ptr, dbl, dbl, ptr, ptr],
    "sumpy_p2p_matrix_subset_f64": [i64, ptr, ptr, ptr, i64, ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_helmholtz_p2p_matrix_subset_f64": [i64, ptr, ptr, ptr, i64, ptr, i64, ptr, dbl, dbl,
                                              ptr, ptr],
    "sumpy_e2p_from_items_grad_mixed": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, i64, dbl,
                                        ptr, ptr, ptr],
    "sumpy_e2p_from_single_box_packed_grad_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr,
                                                  i64, dbl, ptr, ptr, ptr],
    "sumpy_class_gemm_f64": [i32, i32, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr, i32, ptr,
                             i32, ptr, i32, ptr, ptr],
    "sumpy_class_gemm_chain_f64": [i32, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                   ptr, ptr, ptr, ptr, ptr, ptr, ptr],
    "sumpy_class_gemm_tf32x3": [i32, i32, i32, ptr, ptr, ptr, i32, ptr, ptr, ptr, ptr, i32, ptr,
                                ptr, i32, i32, i32, i32, ptr, ptr, i32, ptr, ptr, ptr],
    "sumpy_helmholtz_p2e_from_single_box_levels_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64,
                                                       ptr, ptr, ptr, i64, ptr, ptr, ptr],
    "sumpy_helmholtz_e2p_from_single_box_levels_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64,
                                                       ptr, ptr, ptr, ptr, i64, dbl, ptr, ptr],
    "sumpy_helmholtz_e2p_from_items_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr,
                                           i64, dbl, ptr, ptr],
    "sumpy_helmholtz_p2e_from_items_f64": [cint, dbl, i32, ptr, ptr, ptr, ptr, i64, ptr, i64,
                                           ptr, ptr, ptr],
    "sumpy_e2p_from_items_mixed": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, i64, dbl,
                                   ptr, ptr],
    "sumpy_p2e_from_items_mixed": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, i64, ptr, ptr,
                                   ptr],
    "sumpy_e2p_from_items_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, i64, dbl, ptr,
                                 ptr],
    "sumpy_e2p_from_items_grad_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, ptr, i64, dbl,
                                      ptr, ptr, ptr],
    "sumpy_p2e_from_items_f64": [cint, i32, ptr, ptr, ptr, ptr, i64, ptr, i64, ptr, ptr, ptr],
    # Helmholtz
    "sumpy_helmholtz_p2p_from_csr_f64": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64, dbl,
                                         ptr, ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_helmholtz_p2p_from_csr_mixed": [i32, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, i64,
                                           dbl, ptr, ptr, i64, ptr, dbl, ptr, ptr],
    "sumpy_helmholtz_p2p_direct_f64": [i64, ptr, i64, i64, ptr, i64, dbl, ptr, ptr, dbl, ptr,
                                       ptr],
    "sumpy_helmholtz_p2e_from_single_box_f64": [cint, dbl, dbl, i32, ptr, ptr, i64, ptr, ptr,
                                                ptr, i64, ptr, i32, ptr, ptr],
    "sumpy_helmholtz_e2e_from_children_f64": [cint, cint, dbl, dbl, dbl, i32, ptr, ptr, i64,
                                              ptr, i64, i32, ptr, i32, ptr, ptr],
    "sumpy_helmholtz_e2e_from_parent_f64": [cint, cint, dbl, dbl, dbl, i32, ptr, ptr, ptr, i64,
                                            i32, ptr, i32, ptr, ptr],
    "sumpy_helmholtz_m2l_translation_classes_f64": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                                    ptr, ptr, i32, ptr, i32, ptr, i32, ptr,
                                                    ptr],
    "sumpy_helmholtz_m2l_translation_classes_tf32x3": [cint, i32, ptr, ptr, ptr, i32, ptr, ptr,
                                                       ptr, ptr, i32, ptr, ptr, i32, i32, i32,
                                                       i32, ptr, ptr, i32, ptr, ptr, ptr],
    "sumpy_helmholtz_e2p_from_single_box_f64": [cint, dbl, dbl, i32, ptr, ptr, i64, i32, ptr,
                                                ptr, ptr, ptr, i64, dbl, ptr, ptr],
    "sumpy_helmholtz_e2p_from_csr_f64": [cint, dbl, dbl, i32, ptr, ptr, ptr, ptr, i64, i32,
                                         ptr, ptr, ptr, ptr, i64, dbl, ptr, ptr],
    "sumpy_helmholtz_p2e_from_csr_f64": [cint, dbl, dbl, i32, ptr, ptr, ptr, ptr, i64, ptr,
                                         ptr, ptr, i64, ptr, i32, ptr, ptr],
}

_RESTYPES = {
    "sumpy_version": cint,
    "sumpy_last_error": ctypes.c_char_p,
    "sumpy_get_tc_wait_cycles": i64,
    "sumpy_tree_gpu_free": None,
}

_lib = None


class _LaunchCounter:
    """Counts C-ABI kernel-launching calls (one launch each)."""

    def __init__(self):
        self.value = 0

    def reset(self):
        self.value = 0


launch_counter = _LaunchCounter()


def declare(lib):
    global _lib
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, cint)
    _lib = lib


def exported_names():
    return list(SIGNATURES)


def call(name, *args):
    from sumpy_b200 import _lib as L
    lib = L.load_cuda_library()
    rc = getattr(lib, name)(*args)
    launch_counter.value += 1
    if rc != 0:
        msg = lib.sumpy_last_error().decode()
        raise RuntimeError(f"{name} failed (status {rc}): {msg}")
    return rc


def dptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
