"""Failure detection in the tensor-core kernels, without a GPU fault.

Every barrier wait in the tcgen05 M2L is bounded; a wait that runs out
makes its CTA stop, let its work in flight finish, free its tensor memory
and report status 1 (timeout). The budget is lowered here to a few hundred
cycles, so that the first wait of every CTA expires (a multipole tile
cannot arrive from memory that fast); the launch must still return, report
the timeout through the wrangler's status word, and leave the context
usable: with the default budget restored, the same evaluation is correct.
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
from tests._pointsets import sphere_plummer

pytestmark = pytest.mark.gpu

DEFAULT_CYCLES = 4_000_000_000


def _wrangler(trav, tcls, precision, dev):
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: 8,
                                  translation_classes_data=tcls, precision=precision,
                                  device=dev)


def test_wait_budget_setter_roundtrip(cuda_device):
    from sumpy_b200 import _lib
    L = _lib.load_cuda_library()
    assert L.sumpy_get_tc_wait_cycles() == DEFAULT_CYCLES
    try:
        assert L.sumpy_set_tc_wait_cycles(12345) == 0
        assert L.sumpy_get_tc_wait_cycles() == 12345
    finally:
        L.sumpy_set_tc_wait_cycles(0)
    assert L.sumpy_get_tc_wait_cycles() == DEFAULT_CYCLES


def test_expired_wait_reports_timeout_and_context_survives(cuda_device):
    from sumpy_b200 import _lib
    L = _lib.load_cuda_library()
    dev = cuda_device
    pts = sphere_plummer(8000, 21)
    q = torch.as_tensor(np.random.default_rng(3).standard_normal(8000), device=dev)
    tree, trav, tcls = build_all(pts, None, 24)
    w = _wrangler(trav, tcls, "mixed", dev)
    ref = drive_fmm(None, _wrangler(trav, tcls, "fp64", dev), [q])[0]
    # warm: plans, tables and the module are in place before the budget drops
    drive_fmm(None, w, [q])
    w.check_status()
    try:
        L.sumpy_set_tc_wait_cycles(500)
        drive_fmm(None, w, [q])
        torch.cuda.synchronize()
    finally:
        L.sumpy_set_tc_wait_cycles(0)
    with pytest.raises(RuntimeError, match="wait expired"):
        w.check_status()
    # the context is usable and the status was cleared: a clean evaluation
    (pot,) = drive_fmm(None, w, [q])
    w.check_status()
    err = float((pot - ref).norm() / ref.norm())
    assert err < 1e-5, err


def test_level_chain_wait_expiry_reports_status(cuda_device):
    """The FP64 M2M / L2L run as one persistent launch whose steps wait on
    the previous level; with a budget of a thousand cycles the first unit of
    the second level gives up (the first level's units are still running),
    the launch returns status 2 through the wrangler, and with the default
    budget back the same wrangler evaluates correctly."""
    from oracle import oracle as O
    from sumpy_b200 import _lib
    L = _lib.load_cuda_library()
    dev = cuda_device
    pts = sphere_plummer(20000, 23)
    qn = np.random.default_rng(4).standard_normal(20000)
    q = torch.as_tensor(qn, device=dev)
    tree, trav, tcls = build_all(pts, None, 16)
    w = _wrangler(trav, tcls, "fp64", dev)
    w.chain_levels = True
    drive_fmm(None, w, [q])
    w.check_status()
    try:
        L.sumpy_set_tc_wait_cycles(1000)
        drive_fmm(None, w, [q])
        torch.cuda.synchronize()
    finally:
        L.sumpy_set_tc_wait_cycles(0)
    with pytest.raises(RuntimeError, match="level-chain wait"):
        w.check_status()
    (pot,) = drive_fmm(None, w, [q])
    w.check_status()
    ref = O.run_fmm(tree, trav, tcls, 8, qn, exclude_self=True)
    err = float(np.linalg.norm(pot.cpu().numpy() - ref) / np.linalg.norm(ref))
    assert err < 1e-12, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_level_chain_matches_level_by_level(cuda_device, precision):
    """The chained M2M / L2L launch and the level-by-level launches give the
    same multipoles and locals (FP64 atomics in another order: 1e-13)."""
    dev = cuda_device
    pts = sphere_plummer(30000, 29)
    q = torch.as_tensor(np.random.default_rng(5).standard_normal(30000), device=dev)
    tree, trav, tcls = build_all(pts, None, 20)
    out = {}
    for chain in (True, False):
        w = _wrangler(trav, tcls, precision, dev)
        w.chain_levels = chain
        qs = w.reorder_sources(q)
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                   mp)
        loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                              trav.target_or_target_parent_boxes, loc)
        w.check_status()
        out[chain] = (mp.clone(), loc.clone())
    (mp1, loc1), (mp0, loc0) = out[True], out[False]
    assert float((mp1 - mp0).norm() / mp0.norm()) < 1e-13
    # the mixed form's M2L splits its inputs into TF32 planes: inputs that
    # differ in the last bit may round differently (2^-22 relative at most)
    tol = 1e-13 if precision == "fp64" else 1e-6
    assert float((loc1 - loc0).norm() / loc0.norm()) < tol
