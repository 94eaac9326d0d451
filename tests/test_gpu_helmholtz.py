"""GPU parity for the 3D Helmholtz kernel (G = e^{ikr}/r): each wrangler
stage through the C-ABI against the Helmholtz oracle (pinned to sumpy's own
HelmholtzKernel operators by tests/test_oracle_golden_helmholtz.py), end to
end, the mixed form against the FP64 form, linearity, and convergence in
the order against the direct sum (sumpy/test/test_fmm.py:78-297 runs the
same checks with HelmholtzKernel(3), passing k through kernel_extra_kwargs
and complex128 as the wrangler dtype, test_fmm.py:222-286).

Tolerance: the FP64 GPU stages take the kernel derivatives from the closed
form of sumpy's Tausch recursion (sumpy_b200/csrc/helmholtz.cu), which
agrees with the recursion to ~1e-12 relative at p = 14; parity is asserted
at 1e-11.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sumpy_b200 import (
    P2P,
    HelmholtzKernel,
    LinearPDEConformingVolumeTaylorLocalExpansion as LExp,
    LinearPDEConformingVolumeTaylorMultipoleExpansion as MExp,
    SumpyExpansionWrangler,
    SumpyTreeIndependentDataForWrangler,
    drive_fmm,
)
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer, uniform_cube

pytestmark = pytest.mark.gpu

PARITY = 1e-11
K = 10.0


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def make_wrangler(trav, tcls, order, exclude_self=False, precision="fp64", k=K):
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.complex128, lambda kn, a, t, lev: order,
                                  kernel_extra_kwargs={"k": k},
                                  translation_classes_data=tcls, precision=precision)


def _sphere(n, seed):
    g = np.random.default_rng(seed).standard_normal((3, n))
    return g / np.linalg.norm(g, axis=0)


GEOMS = {
    "uniform_separate": lambda: (uniform_cube(3000, 15), uniform_cube(2000, 18), 30),
    "sphere_self": lambda: (_sphere(4000, 5), None, 24),
    "sphere_plummer_self": lambda: (sphere_plummer(3000, 5), None, 16),
    "sphere_small": lambda: (_sphere(1500, 9), None, 30),
}


def _setup(geom):
    src, tgt, mpb = GEOMS[geom]()
    tree, trav, tcls = build_all(src, tgt, mpb)
    rng = np.random.default_rng(44)
    q = rng.standard_normal(src.shape[1]) + 1j * rng.standard_normal(src.shape[1])
    return src, tgt, tree, trav, tcls, q


@pytest.mark.parametrize("geom", ["uniform_separate", "sphere_self", "sphere_plummer_self"])
@pytest.mark.parametrize("order", [1, 3, 8, 14])
def test_stages_match_oracle(cuda_device, geom, order):
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    stages = {}
    ref = O.run_fmm(tree, trav, tcls, order, q, exclude_self=excl, stages=stages,
                    helmholtz_k=K)

    w = make_wrangler(trav, tcls, order, exclude_self=excl)
    qd = w.reorder_sources(torch.as_tensor(q, device=cuda_device))
    mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
    mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                              trav.source_parent_boxes, mp)
    assert relerr(mp.cpu(), stages["mpoles"]) < PARITY

    pd = w.eval_direct(None, trav.target_boxes, trav.neighbor_source_boxes_starts,
                       trav.neighbor_source_boxes_lists, [qd])
    assert relerr(pd[0].cpu(), stages["pot_direct"]) < PARITY

    loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                               trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
                               trav.from_sep_siblings_lists, mp)
    assert relerr(loc.cpu(), stages["m2l_locals"]) < PARITY

    pm = w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                           trav.from_sep_smaller_by_level, mp)
    if np.any(stages["pot_m2p"]):
        assert relerr(pm[0].cpu(), stages["pot_m2p"]) < PARITY

    pl = w.form_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                       trav.target_or_target_parent_boxes, trav.from_sep_bigger_starts,
                       trav.from_sep_bigger_lists, [qd])
    loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                          trav.target_or_target_parent_boxes, loc + pl)
    assert relerr(loc.cpu(), stages["locals"]) < PARITY

    pe = w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)
    assert relerr(pe[0].cpu(), stages["pot_l2p"]) < PARITY

    (pot,) = drive_fmm(None, w, [torch.as_tensor(q, device=cuda_device)])
    assert relerr(pot.cpu(), ref) < PARITY


def test_high_order_matches_oracle(cuda_device):
    """p = 14 (the order of the 500k-point sphere workload), end to end."""
    src, tgt, tree, trav, tcls, q = _setup("sphere_small")
    ref = O.run_fmm(tree, trav, tcls, 14, q, exclude_self=True, helmholtz_k=K)
    w = make_wrangler(trav, tcls, 14, exclude_self=True)
    (pot,) = drive_fmm(None, w, [torch.as_tensor(q, device=cuda_device)])
    assert relerr(pot.cpu(), ref) < PARITY


def test_p2p_direct_matches_oracle(cuda_device):
    rng = np.random.default_rng(42)
    src = rng.random((3, 3000))
    tgt = rng.random((3, 2000))
    q = rng.standard_normal(3000) + 1j * rng.standard_normal(3000)
    (gpu,) = P2P([HelmholtzKernel(3)])(None, tgt, src, (q,), k=K)
    assert relerr(gpu.cpu(), O.helm_p2p_direct(tgt, src, K, q)) < 1e-13
    (gpu,) = P2P([HelmholtzKernel(3)], exclude_self=True)(
        None, src, src, (q,), target_to_source=np.arange(3000), k=K)
    assert relerr(gpu.cpu(), O.helm_p2p_direct(src, src, K, q, np.arange(3000))) < 1e-13


@pytest.mark.parametrize("geom", ["sphere_self", "uniform_separate"])
def test_converges_against_direct_sum(cuda_device, geom):
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    t = src if excl else tgt
    (ref,) = P2P([HelmholtzKernel(3)], exclude_self=excl)(
        None, t, src, (q,), target_to_source=np.arange(src.shape[1]) if excl else None, k=K)
    errs = []
    for order in (4, 8, 12, 14):
        w = make_wrangler(trav, tcls, order, exclude_self=excl)
        (pot,) = drive_fmm(None, w, [torch.as_tensor(q, device=cuda_device)])
        errs.append(relerr(pot.cpu(), ref.cpu()))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-4, errs


def test_mixed_matches_fp64(cuda_device):
    """Mixed form (complex64 near field on FP64 offsets, split-TF32 M2L on the
    tensor cores) against the FP64 form, stage by stage and end to end.

    The M2L bound is looser than Laplace's: the Helmholtz operators mix
    derivatives of very different magnitude in one class group, and each
    group's products are summed in FP32 on the tensor cores before the FP64
    drain (measured 2.1e-6 on the locals at p = 10; the FP64 FMM's own error
    against the direct sum is of the same size at p = 14)."""
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    qd = torch.as_tensor(q, device=cuda_device)
    wf = make_wrangler(trav, tcls, 10, True)
    wm = make_wrangler(trav, tcls, 10, True, precision="mixed")
    errs = {}
    outs = []
    for w in (wf, wm):
        qs = w.reorder_sources(qd)
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qs])
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        pd = w.eval_direct(None, trav.target_boxes, trav.neighbor_source_boxes_starts,
                           trav.neighbor_source_boxes_lists, [qs])[0]
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                   mp)
        outs.append((pd.cpu(), loc.cpu(), drive_fmm(None, w, [qd])[0].cpu()))
    wm.check_status()
    errs["p2p"] = relerr(outs[1][0], outs[0][0])
    errs["m2l"] = relerr(outs[1][1], outs[0][1])
    errs["total"] = relerr(outs[1][2], outs[0][2])
    assert errs["m2l"] < 5e-6, errs
    assert errs["p2p"] < 1e-6, errs
    assert errs["total"] < 5e-6, errs


def test_linearity_and_k_zero(cuda_device):
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    q2 = np.random.default_rng(7).standard_normal(q.shape) * (1 - 2j)
    w = make_wrangler(trav, tcls, 6, exclude_self=True)
    run = lambda x, ww=w: drive_fmm(None, ww, [torch.as_tensor(x, device=cuda_device)])[0].cpu().numpy()
    a, b = run(q), run(q2)
    ab = run((2.0 + 1j) * q - 3.0 * q2)
    assert relerr(ab, (2.0 + 1j) * a - 3.0 * b) < 1e-12
    # k = 0 reproduces the Laplace FMM on the real and imaginary parts
    from sumpy_b200 import LaplaceKernel
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=True)
    wl = SumpyExpansionWrangler(ti, trav, np.float64, lambda *args: 6,
                                translation_classes_data=tcls)
    h0 = run(q, make_wrangler(trav, tcls, 6, exclude_self=True, k=0.0))
    lr = drive_fmm(None, wl, [torch.as_tensor(q.real, device=cuda_device)])[0].cpu().numpy()
    li = drive_fmm(None, wl, [torch.as_tensor(q.imag, device=cuda_device)])[0].cpu().numpy()
    assert relerr(h0, lr + 1j * li) < 1e-12
