"""The allocation-free tensor-core M2L entry point against the regular one.

``sumpy_m2l_translation_classes_tf32x3_noalloc`` serves callers that cannot
allocate device memory while they run -- for instance a host application
that fixes its device-memory budget at start-up, or an allocation-free
real-time loop. Instead of caller memory it keeps its scratch (the TF32
planes of the source multipoles) in a device array built into the library.

Through the C-ABI, this checks that consecutive calls on different levels
(different sizes and multipoles) give the local expansions that the regular
entry point gives with caller-allocated planes, that a call takes no device
memory, and that a request beyond the built-in capacity is refused with a
clear error. The file is collected last, so that if it fails, a run that stops at
the first failure has already run every other test.
"""
import numpy as np
import pytest
import torch

from sumpy_b200 import (
    LaplaceKernel,
    LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
    LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp,
    SumpyExpansionWrangler,
    SumpyTreeIndependentDataForWrangler,
    _capi,
)
from sumpy_b200.fmm import M2L_TILE, M2L_TILE_TC
from sumpy_b200.tree import build_all
from tests._pointsets import uniform_cube

pytestmark = pytest.mark.gpu

ORDER = 10


def _wrangler_and_multipoles(dev):
    """A small uniform problem, its mixed-form wrangler and its multipoles."""
    tree, trav, _ = build_all(uniform_cube(4000, 15), uniform_cube(3000, 18), 30)
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    w = SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: ORDER,
                               precision="mixed", device=dev)
    q = torch.as_tensor(np.random.default_rng(44).standard_normal(4000), device=dev)
    qd = w.reorder_sources(q)
    mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
    mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                              trav.source_parent_boxes, mp)
    ltb = trav.level_start_target_or_target_parent_box_nrs
    st = trav.from_sep_siblings_starts
    levels = sorted((L for L in range(tree.nlevels)
                     if ltb[L] != ltb[L + 1] and st[ltb[L]] != st[ltb[L + 1]]), reverse=True)
    return w, trav, mp, levels


def _level_inputs(w, trav, mp, lev, tile=M2L_TILE_TC):
    """The tensor-core (or, with tile=M2L_TILE, FP64) schedule of one M2L
    level, built by the wrangler's own planning code, and its operands."""
    dev = w.device
    ltb = trav.level_start_target_or_target_parent_box_nrs
    st = trav.from_sep_siblings_starts
    a, b = int(ltb[lev]), int(ltb[lev + 1])
    plan = w._m2l_plan(lev, trav.target_or_target_parent_boxes[a:b], st[a:b + 1],
                       trav.from_sep_siblings_lists, tile)
    tgs = plan["tile_group_starts"].cpu().numpy()
    it_tile, it_g0, it_g1 = w._tc_items([(int(tgs[i]), int(tgs[i + 1]))
                                         for i in range(plan["ntiles"])])
    mats, mscale = w._m2l_matrices(lev)
    w.tc_format = "tf32"      # the no-alloc entry point takes TF32 planes
    hi, lo, rp, kp, _ = w._m2l_tc_operands(mats)
    sbase, sview = w.multipole_expansions_view(mp, lev)
    tbase, tview = w.local_expansions_view(w.local_expansion_zeros(), lev)
    items = [torch.as_tensor(x).to(dev) for x in (it_tile, it_g0, it_g1)]
    scale = torch.full((plan["ntiles"],), mscale, dtype=torch.float64, device=dev)
    return (plan, items, scale, (hi, lo, rp, kp), sbase, sview.contiguous(), tbase,
            tview.shape, mats)


def _common_args(plan, items, scale, ops):
    hi, lo, rp, kp = ops
    return [_capi.cint(ORDER), _capi.i32(len(items[0])), _capi.dptr(items[0]),
            _capi.dptr(items[1]), _capi.dptr(items[2]), _capi.i32(M2L_TILE_TC),
            _capi.dptr(plan["tile_targets"]), _capi.dptr(scale),
            _capi.dptr(plan["group_class"]), _capi.dptr(plan["group_sources"]),
            _capi.i32(plan["nclasses"]), _capi.dptr(hi), _capi.dptr(lo), _capi.i32(rp),
            _capi.i32(kp)]


def _regular(inp, status):
    """The regular tensor-core entry point with caller-allocated planes."""
    plan, items, scale, ops, sbase, sview, tbase, tshape, _ = inp
    kp = ops[3]
    nb, n = sview.shape
    dev = sview.device
    ws_hi = torch.zeros((nb + 1) * kp, dtype=torch.float32, device=dev)
    ws_lo = torch.zeros_like(ws_hi)
    _capi.call("sumpy_split_tf32x2", _capi.i64(nb), _capi.i32(1), _capi.i32(n),
               _capi.dptr(sview), _capi.i32(1), _capi.i32(kp), _capi.dptr(ws_hi),
               _capi.dptr(ws_lo), _capi.stream_ptr())
    out = torch.zeros(tshape, dtype=torch.float64, device=dev)
    _capi.call("sumpy_m2l_translation_classes_tf32x3", *_common_args(plan, items, scale, ops),
               _capi.i32(nb + 1), _capi.i32(sbase), _capi.dptr(ws_hi), _capi.dptr(ws_lo),
               _capi.i32(tbase), _capi.dptr(out), _capi.dptr(status), _capi.stream_ptr())
    return out


def _no_alloc(inp, out, status):
    plan, items, scale, ops, sbase, sview, tbase, tshape, _ = inp
    _capi.call("sumpy_m2l_translation_classes_tf32x3_noalloc",
               *_common_args(plan, items, scale, ops), _capi.i32(sview.shape[0]),
               _capi.i32(sbase), _capi.dptr(sview), _capi.i32(tbase), _capi.dptr(out),
               _capi.dptr(status), _capi.stream_ptr())


def test_no_alloc_m2l_matches_regular_entry(cuda_device):
    """Three calls in a row -- the deepest M2L level, a coarser level with
    fewer source boxes and other multipoles, the deepest level again -- each
    against the regular entry point (same kernel, so 1e-12: only the order of
    the FP64 atomic additions may differ), the deepest level also against the
    FP64 M2L; no device memory is taken by the second call."""
    dev = cuda_device
    w, trav, mp, levels = _wrangler_and_multipoles(dev)
    assert len(levels) >= 2
    deep = _level_inputs(w, trav, mp, levels[0])
    coarse = _level_inputs(w, trav, mp, levels[1])
    assert coarse[5].shape[0] < deep[5].shape[0]
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    refs = {id(deep): _regular(deep, status), id(coarse): _regular(coarse, status)}

    outs = []
    for k, inp in enumerate((deep, coarse, deep)):
        out = torch.zeros(inp[7], dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _no_alloc(inp, out, status)
        torch.cuda.synchronize()
        if k == 1:
            assert torch.cuda.mem_get_info()[0] == free0
        outs.append((inp, out))
    assert int(status.item()) == 0
    for inp, out in outs:
        ref = refs[id(inp)]
        norm = float(ref.norm())
        assert norm > 0
        assert float((out - ref).norm()) / norm < 1e-12

    # the deepest level against the FP64 M2L on its own (FP64) schedule
    lev = levels[0]
    ltb = trav.level_start_target_or_target_parent_box_nrs
    st = trav.from_sep_siblings_starts
    a, b = int(ltb[lev]), int(ltb[lev + 1])
    plan64 = w._m2l_plan(lev, trav.target_or_target_parent_boxes[a:b], st[a:b + 1],
                         trav.from_sep_siblings_lists, M2L_TILE)
    mats, mscale = w._m2l_matrices(lev)
    items64 = w._level_items(lev, plan64, mscale)
    ref64 = torch.zeros(deep[7], dtype=torch.float64, device=dev)
    w._call_m2l_f64(ORDER, items64, mats, deep[4], deep[5], deep[6], ref64, _capi.stream_ptr())
    torch.cuda.synchronize()
    err = float((outs[0][1] - ref64).norm() / ref64.norm())
    assert err < 1e-5, err


def test_no_alloc_refuses_oversize(cuda_device):
    with pytest.raises(RuntimeError, match="exceeds the built-in scratch"):
        _capi.call("sumpy_m2l_translation_classes_tf32x3_noalloc", _capi.cint(ORDER),
                   _capi.i32(1), None, None, None, _capi.i32(M2L_TILE_TC), None, None, None,
                   None, _capi.i32(316), None, None, _capi.i32(128), _capi.i32(128),
                   _capi.i32(9000), _capi.i32(0), None, _capi.i32(0), None, None,
                   _capi.stream_ptr())
