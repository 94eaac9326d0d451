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
