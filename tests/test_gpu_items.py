"""The one-launch mixed M2P and P2L (work items over all levels,
sumpy_e2p_from_items_mixed / sumpy_p2e_from_items_mixed) against the FP64
stages and the per-level mixed launches they replace, on leaf sizes that give
long List 3 / List 4 (several items per target box) and short ones.

Tolerance: both mixed forms take FP32 derivatives and products on FP64
offsets; per stage they agree with FP64 to ~1e-7 relative (asserted 1e-6).
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
    drive_fmm,
)
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer, uniform_cube

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _wrangler(trav, tcls, order, precision, items, exclude_self):
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=exclude_self)
    w = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order,
                               translation_classes_data=tcls, precision=precision)
    w.item_kernels = items
    return w


def _list3_list4(w, trav, q):
    qd = w.reorder_sources(torch.as_tensor(q, device="cuda"))
    mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
    mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                              trav.source_parent_boxes, mp)
    pm = w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                           trav.from_sep_smaller_by_level, mp)[0]
    pl = w.form_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                       trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                       trav.from_sep_bigger_lists, [qd])
    return pm.cpu().numpy(), pl.cpu().numpy()


@pytest.mark.parametrize("mpb", [8, 40, 96])
@pytest.mark.parametrize("order", [4, 10])
def test_items_match_fp64_and_per_level(cuda_device, mpb, order):
    src = sphere_plummer(40000, 7)
    tree, trav, tcls = build_all(src, None, mpb)
    q = np.random.default_rng(3).standard_normal(src.shape[1])
    f64 = _list3_list4(_wrangler(trav, tcls, order, "fp64", False, True), trav, q)
    lev = _list3_list4(_wrangler(trav, tcls, order, "mixed", False, True), trav, q)
    itm = _list3_list4(_wrangler(trav, tcls, order, "mixed", True, True), trav, q)
    for k in range(2):
        assert np.abs(f64[k]).max() > 0
        assert relerr(itm[k], f64[k]) < 1e-6, (k, relerr(itm[k], f64[k]))
        assert relerr(itm[k], lev[k]) < 1e-6, (k, relerr(itm[k], lev[k]))


@pytest.mark.parametrize("mpb", [8, 96])
@pytest.mark.parametrize("order", [3, 10])
def test_items_fp64_match_per_level(cuda_device, mpb, order):
    """FP64 List 3 / List 4 over work items (sumpy_e2p_from_items_f64,
    sumpy_p2e_from_items_f64) against the per-level FP64 kernels: the same
    FP64 arithmetic summed in another order (asserted 1e-12)."""
    src = sphere_plummer(40000, 9)
    tree, trav, tcls = build_all(src, None, mpb)
    q = np.random.default_rng(8).standard_normal(src.shape[1])
    lev = _list3_list4(_wrangler(trav, tcls, order, "fp64", False, True), trav, q)
    itm = _list3_list4(_wrangler(trav, tcls, order, "fp64", True, True), trav, q)
    for k in range(2):
        assert np.abs(lev[k]).max() > 0
        assert relerr(itm[k], lev[k]) < 1e-12, (k, relerr(itm[k], lev[k]))


def test_items_fp64_gradient_match_per_level(cuda_device):
    src, tgt = sphere_plummer(20000, 17), uniform_cube(12000, 19) * 3.0 - 1.0
    tree, trav, tcls = build_all(src, tgt, 32)
    q = torch.as_tensor(np.random.default_rng(14).standard_normal(src.shape[1]), device="cuda")
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    outs = []
    for new in (False, True):
        w = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: 7, precision="fp64",
                                   translation_classes_data=tcls, gradient=True)
        w.item_kernels = new
        qs = w.reorder_sources(q)
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        pm = w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                               trav.from_sep_smaller_by_level, mp)
        outs.append([t.cpu().numpy() for t in pm])
    for k in range(4):     # potential, d/dx, d/dy, d/dz
        assert np.abs(outs[0][k]).max() > 0
        assert relerr(outs[1][k], outs[0][k]) < 1e-12, k


def test_items_end_to_end_separate_targets(cuda_device):
    src, tgt = uniform_cube(20000, 15), uniform_cube(15000, 18)
    src[:, :5000] *= 0.05          # a dense cluster: long List 3 / List 4
    tree, trav, tcls = build_all(src, tgt, 24)
    q = torch.as_tensor(np.random.default_rng(5).standard_normal(src.shape[1]), device="cuda")
    ref = drive_fmm(None, _wrangler(trav, tcls, 8, "fp64", False, False), [q])[0].cpu()
    w = _wrangler(trav, tcls, 8, "mixed", True, False)
    out = drive_fmm(None, w, [q])[0].cpu()
    w.check_status()
    assert relerr(out, ref) < 2e-6


@pytest.mark.parametrize("order", [1, 3, 10, 16])
def test_merged_p2m_and_packed_l2p_match_per_level(cuda_device, order):
    """P2M of all levels in one launch gives the per-level multipoles bit for
    bit (same per-box arithmetic); the packed L2P agrees with the per-level
    L2P to FP64 rounding; end to end likewise."""
    src, tgt = sphere_plummer(30000, 9), uniform_cube(20000, 4)
    tree, trav, tcls = build_all(src, tgt, 40)
    q = torch.as_tensor(np.random.default_rng(8).standard_normal(src.shape[1]), device="cuda")
    ws = []
    for merged in (False, True):
        w = _wrangler(trav, tcls, order, "fp64", False, False)
        w.merge_levels = merged
        ws.append(w)
    qs = ws[0].reorder_sources(q)
    mps = [w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
           for w in ws]
    assert torch.equal(mps[0], mps[1])
    w = ws[0]
    mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                              trav.source_parent_boxes, mps[0])
    loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                               trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
                               trav.from_sep_siblings_lists, mp)
    loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                          trav.target_or_target_parent_boxes, loc)
    pe = [ww.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)[0].cpu()
          for ww in ws]
    assert np.abs(pe[0].numpy()).max() > 0
    assert relerr(pe[1], pe[0]) < 1e-13
    pots = [drive_fmm(None, ww, [q])[0].cpu() for ww in ws]
    assert relerr(pots[1], pots[0]) < 1e-13


@pytest.mark.parametrize("order", [2, 10])
def test_fp64_gemm_m2m_l2l_match_shift_kernels(cuda_device, order):
    """FP64 form: M2M and L2L as per-octant FP64 GEMMs (the default with one
    order on every level) against the per-box axis-shift kernels."""
    src = sphere_plummer(30000, 12)
    tree, trav, tcls = build_all(src, None, 30)
    q = torch.as_tensor(np.random.default_rng(2).standard_normal(src.shape[1]), device="cuda")
    wg = _wrangler(trav, tcls, order, "fp64", False, True)
    wk = _wrangler(trav, tcls, order, "fp64", False, True)
    wk.gemm_m2m = wk.gemm_l2l = False
    qs = wg.reorder_sources(q)
    mp = wg.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
    outs = []
    for w in (wg, wk):
        m = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                 trav.source_parent_boxes, mp.clone())
        loc = wg.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                    trav.target_or_target_parent_boxes,
                                    trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                    m)
        loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                              trav.target_or_target_parent_boxes, loc)
        outs.append((m.cpu().numpy(), loc.cpu().numpy()))
    assert relerr(outs[0][0], outs[1][0]) < 1e-13
    assert relerr(outs[0][1], outs[1][1]) < 1e-13


@pytest.mark.parametrize("order", [3, 14])
def test_helmholtz_one_launch_stages_match_per_level(cuda_device, order):
    """Helmholtz P2M / L2P of all levels in one launch and List 3 / List 4
    over work items against the per-level launches (FP64, same per-pair
    arithmetic; sums in a different order)."""
    from sumpy_b200 import HelmholtzKernel
    src = sphere_plummer(12000, 31)
    tree, trav, tcls = build_all(src, None, 24)
    rng = np.random.default_rng(6)
    q = torch.as_tensor(rng.standard_normal(src.shape[1]) + 1j * rng.standard_normal(src.shape[1]),
                        device="cuda")
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    outs = []
    for new in (False, True):
        w = SumpyExpansionWrangler(ti, trav, np.complex128, lambda *a: order,
                                   kernel_extra_kwargs={"k": 10.0},
                                   translation_classes_data=tcls)
        w.item_kernels = w.merge_levels = new
        qs = w.reorder_sources(q)
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
        mp2 = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                   trav.source_parent_boxes, mp.clone())
        pm = w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                               trav.from_sep_smaller_by_level, mp2)[0]
        pl = w.form_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                           trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                           trav.from_sep_bigger_lists, [qs])
        pe = w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, pl)[0]
        outs.append([t.cpu().numpy() for t in (mp, pm, pl, pe)])
    for a, b in zip(outs[1], outs[0]):
        assert np.abs(b).max() > 0
        assert relerr(a, b) < 1e-12


@pytest.mark.parametrize("order", [4, 10])
def test_gradient_one_launch_matches_per_level(cuda_device, order):
    """Gradient outputs (the adjoint's position gradients): List 3 over work
    items (mixed) and the packed L2P (FP64) against the per-level kernels."""
    src, tgt = sphere_plummer(20000, 13), uniform_cube(15000, 21) * 3.0 - 1.0
    tree, trav, tcls = build_all(src, tgt, 32)
    q = torch.as_tensor(np.random.default_rng(12).standard_normal(src.shape[1]), device="cuda")
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    outs = []
    for new in (False, True):
        w = SumpyExpansionWrangler(ti, trav, np.float64, lambda *a: order, precision="mixed",
                                   translation_classes_data=tcls, gradient=True)
        w.item_kernels = w.merge_levels = new
        qs = w.reorder_sources(q)
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        pm = w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                               trav.from_sep_smaller_by_level, mp)
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                   mp)
        pe = w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)
        outs.append(([t.cpu().numpy() for t in pm], [t.cpu().numpy() for t in pe]))
    for k in range(4):     # potential, d/dx, d/dy, d/dz
        assert np.abs(outs[0][0][k]).max() > 0
        assert relerr(outs[1][0][k], outs[0][0][k]) < 1e-6, k
        assert relerr(outs[1][1][k], outs[0][1][k]) < 1e-12, k


@pytest.mark.parametrize("order", [2, 9, 14, 16])
def test_helmholtz_packed_l2p_matches_per_box(cuda_device, order):
    """Helmholtz L2P over packed items (several boxes per warp, layout
    decompression with each box's own kappa) against the warp-per-box L2P."""
    from sumpy_b200 import HelmholtzKernel
    src, tgt = sphere_plummer(15000, 41), uniform_cube(9000, 42) * 2.0 - 0.5
    tree, trav, tcls = build_all(src, tgt, 20)
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl])
    rng = np.random.default_rng(43)
    outs = []
    for packed in (False, True):
        w = SumpyExpansionWrangler(ti, trav, np.complex128, lambda *a: order,
                                   kernel_extra_kwargs={"k": 7.0},
                                   translation_classes_data=tcls)
        w.packed_l2p = packed
        loc = torch.as_tensor(
            rng.standard_normal(w.local_expansion_zeros().numel()) * (1 + 0.5j), device="cuda")
        rng = np.random.default_rng(43)   # the same locals for both
        pe = w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)[0]
        outs.append(pe.cpu().numpy())
    assert np.abs(outs[0]).max() > 0
    assert relerr(outs[1], outs[0]) < 1e-12
