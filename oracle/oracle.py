"""ctypes front end of the FP64 CPU oracle (``oracle/fmm_oracle.c`` for
Laplace, ``oracle/helmholtz_oracle.c`` for Helmholtz).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by the smoke check in
``__graft_entry__.py`` and by the CPU-baseline / reference arm of
``bench.py``. The product package ``sumpy_b200`` never imports it.

Point-level functions restate sumpy's individual operators; :func:`run_fmm`
strings the stage-level functions together in boxtree's ``drive_fmm`` order
(the sequence listed in sumpy's wrangler, ``sumpy/fmm.py:609-1086``) over a
tree and traversal produced by :mod:`sumpy_b200.tree`.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle_fmm.so"
_lib = None

_d = ctypes.c_double
_i = ctypes.c_int
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_p = ctypes.c_void_p


def build() -> Path:
    """Compile the oracle library in place (``make`` in ``oracle/``)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        _lib.oracle_l2p_point.restype = _d
        _lib.oracle_m2p_point.restype = _d
    return _lib


def num_threads() -> int:
    """OpenMP threads the oracle's parallel regions use."""
    return int(lib().oracle_num_threads())


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle needs contiguous arrays"
    return a.ctypes.data_as(_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32a(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# {{{ coefficient sets

def ncoeff(p: int) -> int:
    return (p + 1) ** 2


def stored_ids(p: int) -> np.ndarray:
    out = np.zeros((ncoeff(p), 3), dtype=np.int32)
    lib().oracle_stored_ids(_i(p), _ptr(out))
    return out


def full_ids(p: int) -> np.ndarray:
    out = np.zeros(((p + 1) * (p + 2) * (p + 3) // 6, 3), dtype=np.int32)
    lib().oracle_full_ids(_i(p), _ptr(out))
    return out

# }}}


# {{{ point-level operators (no kernel scaling)

def p2m(p, rscale, center, sources, strengths):
    s = _f64(sources)
    q = _f64(strengths)
    out = np.zeros(ncoeff(p))
    lib().oracle_p2m_point(_i(p), _d(rscale), _ptr(_f64(center)), _i(s.shape[1]),
                           _ptr(_f64(s[0])), _ptr(_f64(s[1])), _ptr(_f64(s[2])),
                           _ptr(q), _ptr(out))
    return out


def p2l(p, rscale, center, sources, strengths):
    s = _f64(sources)
    q = _f64(strengths)
    out = np.zeros(ncoeff(p))
    lib().oracle_p2l_point(_i(p), _d(rscale), _ptr(_f64(center)), _i(s.shape[1]),
                           _ptr(_f64(s[0])), _ptr(_f64(s[1])), _ptr(_f64(s[2])),
                           _ptr(q), _ptr(out))
    return out


def l2p(p, rscale, coeffs, bvec):
    return lib().oracle_l2p_point(_i(p), _d(rscale), _ptr(_f64(coeffs)),
                                  _ptr(_f64(bvec)))


def m2p(p, rscale, coeffs, bvec):
    return lib().oracle_m2p_point(_i(p), _d(rscale), _ptr(_f64(coeffs)),
                                  _ptr(_f64(bvec)))


def m2m(psrc, ptgt, rsrc, rtgt, dvec, coeffs):
    out = np.zeros(ncoeff(ptgt))
    lib().oracle_m2m_point(_i(psrc), _i(ptgt), _d(rsrc), _d(rtgt),
                           _ptr(_f64(dvec)), _ptr(_f64(coeffs)), _ptr(out))
    return out


def l2l(psrc, ptgt, rsrc, rtgt, dvec, coeffs):
    out = np.zeros(ncoeff(ptgt))
    lib().oracle_l2l_point(_i(psrc), _i(ptgt), _d(rsrc), _d(rtgt),
                           _ptr(_f64(dvec)), _ptr(_f64(coeffs)), _ptr(out))
    return out


def m2l(p, rsrc, rtgt, dvec, coeffs):
    out = np.zeros(ncoeff(p))
    lib().oracle_m2l_point(_i(p), _d(rsrc), _d(rtgt), _ptr(_f64(dvec)),
                           _ptr(_f64(coeffs)), _ptr(out))
    return out

# }}}


# {{{ Helmholtz point-level operators (helmholtz_oracle.c; complex128)

def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def helm_p2m(p, rscale, k, center, sources, strengths):
    s = _f64(sources)
    q = _c128(strengths)
    out = np.zeros(ncoeff(p), dtype=np.complex128)
    lib().oracle_helm_p2m_point(_i(p), _d(rscale), _d(k), _ptr(_f64(center)),
                                _i(s.shape[1]), _ptr(_f64(s[0])), _ptr(_f64(s[1])),
                                _ptr(_f64(s[2])), _ptr(q), _ptr(out))
    return out


def helm_p2l(p, rscale, k, center, sources, strengths):
    s = _f64(sources)
    q = _c128(strengths)
    out = np.zeros(ncoeff(p), dtype=np.complex128)
    lib().oracle_helm_p2l_point(_i(p), _d(rscale), _d(k), _ptr(_f64(center)),
                                _i(s.shape[1]), _ptr(_f64(s[0])), _ptr(_f64(s[1])),
                                _ptr(_f64(s[2])), _ptr(q), _ptr(out))
    return out


def helm_l2p(p, rscale, k, coeffs, bvec):
    out = np.zeros(1, dtype=np.complex128)
    lib().oracle_helm_l2p_point(_i(p), _d(rscale), _d(k), _ptr(_c128(coeffs)),
                                _ptr(_f64(bvec)), _ptr(out))
    return out[0]


def helm_m2p(p, rscale, k, coeffs, bvec):
    out = np.zeros(1, dtype=np.complex128)
    lib().oracle_helm_m2p_point(_i(p), _d(rscale), _d(k), _ptr(_c128(coeffs)),
                                _ptr(_f64(bvec)), _ptr(out))
    return out[0]


def helm_m2m(psrc, ptgt, rsrc, rtgt, k, dvec, coeffs):
    out = np.zeros(ncoeff(ptgt), dtype=np.complex128)
    lib().oracle_helm_m2m_point(_i(psrc), _i(ptgt), _d(rsrc), _d(rtgt), _d(k),
                                _ptr(_f64(dvec)), _ptr(_c128(coeffs)), _ptr(out))
    return out


def helm_l2l(psrc, ptgt, rsrc, rtgt, k, dvec, coeffs):
    out = np.zeros(ncoeff(ptgt), dtype=np.complex128)
    lib().oracle_helm_l2l_point(_i(psrc), _i(ptgt), _d(rsrc), _d(rtgt), _d(k),
                                _ptr(_f64(dvec)), _ptr(_c128(coeffs)), _ptr(out))
    return out


def helm_m2l(p, rsrc, rtgt, k, dvec, coeffs):
    out = np.zeros(ncoeff(p), dtype=np.complex128)
    lib().oracle_helm_m2l_point(_i(p), _d(rsrc), _d(rtgt), _d(k), _ptr(_f64(dvec)),
                                _ptr(_c128(coeffs)), _ptr(out))
    return out


def helm_derivs(x, rscale, k, maxdeg):
    """D[i][j][l] = rscale^|mi| d^mi (e^{ikr}/r) at x for mi0 <= 1, |mi| <= maxdeg."""
    out = np.zeros((2, maxdeg + 1, maxdeg + 1), dtype=np.complex128)
    lib().oracle_helm_derivs(_ptr(_f64(x)), _d(rscale), _d(k), _i(maxdeg), _ptr(out))
    return out


def helm_p2p_direct(targets, sources, k, strengths, target_to_source=None):
    """FP64 direct sum 1/(4 pi) sum_s q_s e^{ik|t-s|}/|t-s| (complex strengths)."""
    t = _f64(targets)
    s = _f64(sources)
    q = _c128(strengths)
    pot = np.zeros(t.shape[1], dtype=np.complex128)
    tts = None if target_to_source is None else _i32a(target_to_source)
    tx, ty, tz = (_f64(t[i]) for i in range(3))
    sx, sy, sz = (_f64(s[i]) for i in range(3))
    lib().oracle_helm_p2p_direct(_i64(t.shape[1]), _ptr(tx), _ptr(ty), _ptr(tz),
                                 _i64(s.shape[1]), _ptr(sx), _ptr(sy), _ptr(sz), _d(k),
                                 _ptr(q), _ptr(tts), _ptr(pot))
    return pot

# }}}


# {{{ direct sum

def p2p_direct(targets, sources, strengths, target_to_source=None):
    """FP64 direct sum 1/(4 pi) sum_s q_s/|t-s| (OpenMP over targets)."""
    t = _f64(targets)
    s = _f64(sources)
    q = _f64(strengths)
    pot = np.zeros(t.shape[1])
    tts = None if target_to_source is None else _i32a(target_to_source)
    tx, ty, tz = (_f64(t[i]) for i in range(3))
    sx, sy, sz = (_f64(s[i]) for i in range(3))
    lib().oracle_p2p_direct(_i64(t.shape[1]), _ptr(tx), _ptr(ty), _ptr(tz),
                            _i64(s.shape[1]), _ptr(sx), _ptr(sy), _ptr(sz),
                            _ptr(q), _ptr(tts), _ptr(pot))
    return pot

# }}}


# {{{ interaction matrix entries

def p2p_matrix_entries(targets, sources, tgtindices, srcindices, target_to_source=None,
                       helmholtz_k=None):
    """FP64 entries G(t - s) / (4 pi) at index pairs, numpy: the arithmetic of
    sumpy's P2PMatrixSubsetGenerator (sumpy/p2p.py:354-477: d = targets[itgt]
    - sources[isrc], p2p.py:392-397) with the kernel expressions of
    LaplaceKernel(3) (1/r) or HelmholtzKernel(3) (e^{ikr}/r) and their
    global scaling 1/(4 pi) (sumpy/kernel.py:639-691, 754-844); with
    target_to_source the pairs with isrc == target_to_source[itgt] are 0
    (p2p.py:162-170, 397-398). The dense P2PMatrixGenerator
    (p2p.py:290-349) is the subset of all pairs."""
    t = np.asarray(targets, dtype=np.float64)
    s = np.asarray(sources, dtype=np.float64)
    it = np.asarray(tgtindices, dtype=np.int64)
    js = np.asarray(srcindices, dtype=np.int64)
    d = t[:, it] - s[:, js]
    r = np.sqrt((d * d).sum(axis=0))
    self_pair = np.zeros(len(it), dtype=bool)
    if target_to_source is not None:
        self_pair = np.asarray(target_to_source, dtype=np.int64)[it] == js
    r = np.where(self_pair, 1.0, r)
    if helmholtz_k is None:
        val = 1.0 / r
    else:
        val = np.exp(1j * helmholtz_k * r) / r
    return np.where(self_pair, 0.0, val) / (4 * np.pi)


def p2p_matrix(targets, sources, target_to_source=None, helmholtz_k=None):
    """The dense [ntargets, nsources] matrix of p2p_matrix_entries."""
    nt = np.asarray(targets).shape[1]
    ns = np.asarray(sources).shape[1]
    it, js = np.meshgrid(np.arange(nt), np.arange(ns), indexing="ij")
    return p2p_matrix_entries(targets, sources, it.ravel(), js.ravel(), target_to_source,
                              helmholtz_k).reshape(nt, ns)

# }}}


# {{{ whole FMM over a tree

def run_fmm(tree, trav, tcls, order, weights, exclude_self=False,
            rscale_fn=None, stages=None, helmholtz_k=None):
    """FP64 FMM in boxtree ``drive_fmm`` order, on host numpy arrays.

    :arg tree, trav, tcls: host objects from :mod:`sumpy_b200.tree`
        (tree, traversal, translation classes).
    :arg order: expansion order (same on every level).
    :arg weights: strengths in *user* source order.
    :arg stages: optional dict; when given, intermediate arrays are stored
        into it (``mpoles``, ``locals``, per-stage potentials) for stage-level
        comparisons.
    :arg helmholtz_k: run the Helmholtz oracle (``helmholtz_oracle.c``,
        G = e^{ikr}/r, complex strengths and results) with this wave number.
    :returns: potentials in user target order.
    """
    L = lib()
    H = helmholtz_k is not None
    kk = [_d(helmholtz_k)] if H else []
    dt = np.complex128 if H else np.float64

    def fn(name):
        return getattr(L, ("oracle_helm_" if H else "oracle_") + name)
    p = order
    nc = ncoeff(p)
    nlev = tree.nlevels
    lsb = np.asarray(tree.level_start_box_nrs, dtype=np.int64)
    cx, cy, cz = (_f64(tree.box_centers[i]) for i in range(3))
    sx, sy, sz = (_f64(tree.sources[i]) for i in range(3))
    tx, ty, tz = (_f64(tree.targets[i]) for i in range(3))
    bss = _i32a(tree.box_source_starts)
    bsc = _i32a(tree.box_source_counts_nonchild)
    bts = _i32a(tree.box_target_starts)
    btc = _i32a(tree.box_target_counts_nonchild)
    child = _i32a(tree.box_child_ids)
    parent = _i32a(tree.box_parent_ids)

    def rscale(lev):
        if rscale_fn is not None:
            return rscale_fn(lev)
        return tree.root_extent * 2.0 ** (-lev) * 2.0 / p

    q = np.ascontiguousarray(np.asarray(weights)[tree.user_source_ids], dtype=dt)
    tts = None
    if exclude_self:
        tts = _i32a(tree.target_to_source)

    mpoles = np.zeros(tree.nboxes * nc, dtype=dt)
    locs = np.zeros(tree.nboxes * nc, dtype=dt)

    def lview(arr, lev):
        return arr[lsb[lev] * nc:lsb[lev + 1] * nc]

    # form_multipoles
    lss = trav.level_start_source_box_nrs
    for lev in range(nlev):
        a, b = lss[lev], lss[lev + 1]
        if a == b:
            continue
        boxes = _i32a(trav.source_boxes[a:b])
        fn("p2m_level")(_i(p), _d(rscale(lev)), *kk, _i32(b - a), _ptr(boxes),
                           _i32(lsb[lev]), _ptr(cx), _ptr(cy), _ptr(cz),
                           _ptr(bss), _ptr(bsc), _ptr(sx), _ptr(sy), _ptr(sz),
                           _ptr(q), _ptr(lview(mpoles, lev)))
    # coarsen_multipoles
    lsp = trav.level_start_source_parent_box_nrs
    for src_lev in range(nlev - 1, 2, -1):
        tgt_lev = src_lev - 1
        a, b = lsp[tgt_lev], lsp[tgt_lev + 1]
        if a == b:
            continue
        boxes = _i32a(trav.source_parent_boxes[a:b])
        fn("m2m_level")(_i(p), _i(p), _d(rscale(src_lev)), _d(rscale(tgt_lev)), *kk,
                           _i32(b - a), _ptr(boxes), _ptr(child), _i64(child.shape[1]),
                           _ptr(cx), _ptr(cy), _ptr(cz),
                           _i32(lsb[src_lev]), _ptr(lview(mpoles, src_lev)),
                           _i32(lsb[tgt_lev]), _ptr(lview(mpoles, tgt_lev)))
    if stages is not None:
        stages["mpoles"] = mpoles.copy()

    # eval_direct (List 1)
    pot_direct = np.zeros(tree.ntargets, dtype=dt)
    tb = _i32a(trav.target_boxes)
    if len(tb):
        fn("p2p_csr")(_i32(len(tb)), _ptr(tb), _ptr(_i32a(trav.neighbor_source_boxes_starts)),
                         _ptr(_i32a(trav.neighbor_source_boxes_lists)),
                         _ptr(bss), _ptr(bsc), _ptr(bts), _ptr(btc),
                         _ptr(sx), _ptr(sy), _ptr(sz), *kk, _ptr(q),
                         _ptr(tx), _ptr(ty), _ptr(tz), _ptr(tts), _ptr(pot_direct))

    # multipole_to_local (List 2)
    ltt = trav.level_start_target_or_target_parent_box_nrs
    tpb = trav.target_or_target_parent_boxes
    s2s = trav.from_sep_siblings_starts
    s2l = _i32a(trav.from_sep_siblings_lists)
    ecls = _i32a(tcls.from_sep_siblings_translation_classes)
    cvec = _f64(tcls.from_sep_siblings_translation_class_to_distance_vector)
    cls_ls = tcls.from_sep_siblings_translation_classes_level_starts
    m2l_locs = np.zeros_like(locs)
    for lev in range(nlev):
        a, b = ltt[lev], ltt[lev + 1]
        if a == b or s2s[a] == s2s[b]:
            continue
        boxes = _i32a(tpb[a:b])
        starts = _i32a(np.asarray(s2s[a:b + 1]))
        fn("m2l_level")(_i(p), _d(rscale(lev)), *kk, _i32(b - a), _ptr(boxes),
                           _ptr(starts), _ptr(s2l), _ptr(ecls),
                           _i32(cls_ls[lev + 1] - cls_ls[lev]), _i32(cls_ls[lev]),
                           _ptr(cvec), _i64(cvec.shape[1]), _i32(lsb[lev]),
                           _ptr(lview(mpoles, lev)), _ptr(lview(m2l_locs, lev)))
    if stages is not None:
        stages["m2l_locals"] = m2l_locs.copy()

    # eval_multipoles (List 3)
    pot_m2p = np.zeros(tree.ntargets, dtype=dt)
    for lev in range(nlev):
        tgt = trav.target_boxes_sep_smaller_by_source_level[lev]
        if len(tgt) == 0:
            continue
        lst = trav.from_sep_smaller_by_level[lev]
        fn("m2p_level")(_i(p), _d(rscale(lev)), *kk, _i32(len(tgt)), _ptr(_i32a(tgt)),
                           _ptr(_i32a(lst.starts)), _ptr(_i32a(lst.lists)),
                           _ptr(cx), _ptr(cy), _ptr(cz), _i32(lsb[lev]),
                           _ptr(lview(mpoles, lev)), _ptr(bts), _ptr(btc),
                           _ptr(tx), _ptr(ty), _ptr(tz), _ptr(pot_m2p))

    # form_locals (List 4)
    p2l_locs = np.zeros_like(locs)
    s4s = trav.from_sep_bigger_starts
    s4l = _i32a(trav.from_sep_bigger_lists)
    for lev in range(nlev):
        a, b = ltt[lev], ltt[lev + 1]
        if a == b:
            continue
        boxes = _i32a(tpb[a:b])
        starts = _i32a(np.asarray(s4s[a:b + 1]))
        fn("p2l_level")(_i(p), _d(rscale(lev)), *kk, _i32(b - a), _ptr(boxes),
                           _ptr(starts), _ptr(s4l), _ptr(cx), _ptr(cy), _ptr(cz),
                           _ptr(bss), _ptr(bsc), _ptr(sx), _ptr(sy), _ptr(sz),
                           _ptr(q), _i32(lsb[lev]), _ptr(lview(p2l_locs, lev)))
    locs = m2l_locs + p2l_locs

    # refine_locals
    for tgt_lev in range(1, nlev):
        a, b = ltt[tgt_lev], ltt[tgt_lev + 1]
        if a == b:
            continue
        src_lev = tgt_lev - 1
        boxes = _i32a(tpb[a:b])
        fn("l2l_level")(_i(p), _i(p), _d(rscale(src_lev)), _d(rscale(tgt_lev)), *kk,
                           _i32(b - a), _ptr(boxes), _ptr(parent),
                           _ptr(cx), _ptr(cy), _ptr(cz),
                           _i32(lsb[src_lev]), _ptr(lview(locs, src_lev)),
                           _i32(lsb[tgt_lev]), _ptr(lview(locs, tgt_lev)))
    if stages is not None:
        stages["locals"] = locs.copy()

    # eval_locals
    pot_l2p = np.zeros(tree.ntargets, dtype=dt)
    ltb = trav.level_start_target_box_nrs
    for lev in range(nlev):
        a, b = ltb[lev], ltb[lev + 1]
        if a == b:
            continue
        boxes = _i32a(trav.target_boxes[a:b])
        fn("l2p_level")(_i(p), _d(rscale(lev)), *kk, _i32(b - a), _ptr(boxes),
                           _ptr(cx), _ptr(cy), _ptr(cz), _i32(lsb[lev]),
                           _ptr(lview(locs, lev)), _ptr(bts), _ptr(btc),
                           _ptr(tx), _ptr(ty), _ptr(tz), _ptr(pot_l2p))

    if stages is not None:
        stages["pot_direct"] = pot_direct
        stages["pot_m2p"] = pot_m2p
        stages["pot_l2p"] = pot_l2p
    pot = pot_direct + pot_m2p + pot_l2p
    return pot[tree.sorted_target_ids]

# }}}
