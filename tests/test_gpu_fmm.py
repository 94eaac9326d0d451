"""GPU parity: each wrangler stage through the C-ABI against the FP64 oracle.

Mirrors sumpy's tests: the FP64 form must agree with the CPU restatement of
sumpy's algorithm to 1e-12 relative (stage by stage and end to end),
converge in the order against the direct sum (test_sumpy_fmm,
sumpy/test/test_fmm.py:78-297), be linear in the strengths to 1e-12
(test_unified_single_and_double, test_fmm.py:386-469), and handle
exclude_self (test_fmm.py:538-598).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sumpy_b200 import (
    P2P,
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

PARITY = 1e-12


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def make_wrangler(tree, trav, order, exclude_self=False, precision="fp64"):
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: order,
                                  precision=precision)


GEOMS = {
    "uniform_separate": lambda: (uniform_cube(4000, 15), uniform_cube(3000, 18), 30),
    "sphere_plummer_self": lambda: (sphere_plummer(5000, 5), None, 16),
}


def _setup(geom):
    src, tgt, mpb = GEOMS[geom]()
    tree, trav, tcls = build_all(src, tgt, mpb)
    q = np.random.default_rng(44).standard_normal(src.shape[1])
    return src, tgt, tree, trav, tcls, q


@pytest.mark.parametrize("geom", list(GEOMS))
@pytest.mark.parametrize("order", [1, 3, 6, 10, 16])
def test_stages_match_oracle(cuda_device, geom, order):
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    stages = {}
    ref = O.run_fmm(tree, trav, tcls, order, q, exclude_self=excl, stages=stages)

    w = make_wrangler(tree, trav, order, exclude_self=excl)
    qd = w.reorder_sources(torch.as_tensor(q, device=cuda_device))
    (qd,) = w.distribute_source_weights([qd])
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


def test_p2p_direct_matches_oracle(cuda_device):
    rng = np.random.default_rng(42)
    src = rng.random((3, 3000))
    tgt = rng.random((3, 2000))
    q = rng.random(3000)
    (gpu,) = P2P([LaplaceKernel(3)])(None, tgt, src, (q,))
    assert relerr(gpu.cpu(), O.p2p_direct(tgt, src, q)) < 1e-14
    (gpu,) = P2P([LaplaceKernel(3)], exclude_self=True)(
        None, src, src, (q,), target_to_source=np.arange(3000))
    assert relerr(gpu.cpu(), O.p2p_direct(src, src, q, np.arange(3000))) < 1e-14


@pytest.mark.parametrize("geom", list(GEOMS))
def test_fmm_converges_against_direct_sum(cuda_device, geom):
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    t = src if excl else tgt
    (ref,) = P2P([LaplaceKernel(3)], exclude_self=excl)(
        None, t, src, (q,), target_to_source=np.arange(src.shape[1]) if excl else None)
    errs = []
    for order in (2, 4, 6, 8):
        w = make_wrangler(tree, trav, order, exclude_self=excl)
        (pot,) = drive_fmm(None, w, [torch.as_tensor(q, device=cuda_device)])
        errs.append(relerr(pot.cpu(), ref.cpu()))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-4


def test_linearity(cuda_device):
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    q2 = np.random.default_rng(7).standard_normal(q.shape)
    w = make_wrangler(tree, trav, 6, exclude_self=True)
    run = lambda x: drive_fmm(None, w, [torch.as_tensor(x, device=cuda_device)])[0].cpu().numpy()
    a, b = run(q), run(q2)
    ab = run(2.0 * q - 3.0 * q2)
    assert relerr(ab, 2.0 * a - 3.0 * b) < 1e-12


def test_mixed_precision_accuracy(cuda_device):
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    (ref,) = P2P([LaplaceKernel(3)], exclude_self=True)(
        None, src, src, (q,), target_to_source=np.arange(src.shape[1]))
    w64 = make_wrangler(tree, trav, 10, exclude_self=True)
    wmx = make_wrangler(tree, trav, 10, exclude_self=True, precision="mixed")
    qd = torch.as_tensor(q, device=cuda_device)
    e64 = relerr(drive_fmm(None, w64, [qd])[0].cpu(), ref.cpu())
    emx = relerr(drive_fmm(None, wmx, [qd])[0].cpu(), ref.cpu())
    wmx.check_status()
    # FP32 rounding must stay well below the order-10 truncation error
    assert emx < max(1.2 * e64, 1e-6), (e64, emx)


def test_single_box_tree(cuda_device):
    rng = np.random.default_rng(1)
    src = rng.random((3, 20))
    tgt = rng.random((3, 7))
    q = rng.standard_normal(20)
    tree, trav, tcls = build_all(src, tgt, 30)
    w = make_wrangler(tree, trav, 4)
    (pot,) = drive_fmm(None, w, [torch.as_tensor(q, device=cuda_device)])
    assert relerr(pot.cpu(), O.p2p_direct(tgt, src, q)) < 1e-14


def test_bad_arguments_raise(cuda_device):
    from sumpy_b200 import _capi
    with pytest.raises(RuntimeError, match="unsupported order"):
        _capi.call("sumpy_p2e_from_single_box_f64", _capi.cint(40), _capi.dbl(1.0),
                   _capi.i32(1), None, None, _capi.i64(0), None, None, None, _capi.i64(0),
                   None, _capi.i32(0), None, None)
    with pytest.raises(RuntimeError, match="null pointer"):
        _capi.call("sumpy_p2p_from_csr_f64", _capi.i32(3), None, None, None, None, None,
                   None, None, None, _capi.i64(0), None, None, _capi.i64(0), None,
                   _capi.dbl(1.0), None, None)


def test_split_tf32x2(cuda_device):
    from sumpy_b200 import _capi
    x = torch.randn(3, 5, 7, dtype=torch.float64, device=cuda_device) * 1e3
    hi = torch.empty(3, 8, 32, dtype=torch.float32, device=cuda_device)
    lo = torch.empty_like(hi)
    _capi.call("sumpy_split_tf32x2", _capi.i64(3), _capi.i32(5), _capi.i32(7),
               _capi.dptr(x), _capi.i32(8), _capi.i32(32), _capi.dptr(hi), _capi.dptr(lo),
               _capi.stream_ptr())
    torch.cuda.synchronize()
    bits_hi = hi.view(torch.int32) & 0x1FFF
    bits_lo = lo.view(torch.int32) & 0x1FFF
    assert int(bits_hi.abs().sum()) == 0 and int(bits_lo.abs().sum()) == 0  # TF32-exact
    rec = hi[:, :5, :7].double() + lo[:, :5, :7].double()
    assert float(((rec - x).abs() / x.abs()).max()) < 2.0 ** -21
    assert float(hi[:, 5:, :].abs().sum() + hi[:, :, 7:].abs().sum()) == 0.0


def test_split_f16x2_rowscale(cuda_device):
    """Rows of very different magnitudes: each scaled by a power of two into
    [2^13, 2^14) and split into two f16 halves that restore it to ~2^-22."""
    from sumpy_b200 import _capi
    g = torch.Generator(device="cpu").manual_seed(3)
    mags = 10.0 ** torch.linspace(-30, 30, 3 * 6, dtype=torch.float64).reshape(3, 6, 1)
    x = (torch.randn(3, 6, 7, dtype=torch.float64, generator=g) * mags).to(cuda_device)
    x[1, 2] = 0.0
    hi = torch.empty(3, 8, 64, dtype=torch.float16, device=cuda_device)
    lo = torch.empty_like(hi)
    inv = torch.empty(3, 8, dtype=torch.float32, device=cuda_device)
    _capi.call("sumpy_split_f16x2_rowscale", _capi.i64(3), _capi.i32(6), _capi.i32(7),
               _capi.dptr(x), _capi.i32(8), _capi.i32(64), _capi.dptr(hi), _capi.dptr(lo),
               _capi.dptr(inv), _capi.stream_ptr())
    torch.cuda.synchronize()
    mant, _ = torch.frexp(inv)
    assert bool((mant == 0.5).all())                               # powers of two
    rec = (hi[:, :6, :7].double() + lo[:, :6, :7].double()) * inv[:, :6, None].double()
    rowmax = x.abs().amax(dim=2, keepdim=True).clamp_min(1e-300)
    assert float(((rec - x).abs() / rowmax).max()) < 2.0 ** -21
    scaled = hi[:, :6, :7].double().abs().amax(dim=2)
    nz = x.abs().amax(dim=2) > 0
    assert bool(((scaled[nz] >= 2.0 ** 13 * (1 - 2 ** -10)) & (scaled[nz] <= 2.0 ** 14)).all())
    assert float(inv[1, 2]) == 1.0 and float(hi[1, 2].abs().sum()) == 0.0
    assert float(hi[:, 6:].abs().sum() + hi[:, :, 7:].abs().sum()) == 0.0
    assert bool((inv[:, 6:] == 1.0).all())


@pytest.mark.parametrize("fmt", ["f16", "tf32"])
@pytest.mark.parametrize("geom", list(GEOMS))
@pytest.mark.parametrize("order", [4, 10])
def test_tensor_core_m2l_matches_fp64(cuda_device, geom, order, fmt):
    """3xF16 (row-scaled) and 3xTF32 tcgen05 M2L against the FP64 GEMM on the
    same multipoles."""
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    w64 = make_wrangler(tree, trav, order, exclude_self=excl)
    wtc = make_wrangler(tree, trav, order, exclude_self=excl, precision="mixed")
    wtc.tc_format = fmt
    qd = w64.reorder_sources(torch.as_tensor(q, device=cuda_device))
    mp = w64.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
    mp = w64.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                trav.source_parent_boxes, mp)
    args = (None, trav.level_start_target_or_target_parent_box_nrs,
            trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
            trav.from_sep_siblings_lists, mp)
    l64 = w64.multipole_to_local(*args)
    ltc = wtc.multipole_to_local(*args)
    wtc.check_status()
    err = relerr(ltc.cpu(), l64.cpu())
    assert err < 2e-6, err


def test_mixed_fmm_matches_fp64_fmm(cuda_device):
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    qd = torch.as_tensor(q, device=cuda_device)
    w64 = make_wrangler(tree, trav, 8, exclude_self=True)
    wmx = make_wrangler(tree, trav, 8, exclude_self=True, precision="mixed")
    p64 = drive_fmm(None, w64, [qd])[0].cpu()
    pmx = drive_fmm(None, wmx, [qd])[0].cpu()
    wmx.check_status()
    assert relerr(pmx, p64) < 1e-6


def test_tensor_core_m2l_scale_invariant(cuda_device):
    """Strengths scaled by 1e-30 and 1e30: the row-scaled f16 M2L keeps the
    same relative accuracy (no f16 underflow or overflow)."""
    src, tgt, tree, trav, tcls, q = _setup("sphere_plummer_self")
    w64 = make_wrangler(tree, trav, 8, exclude_self=True)
    wtc = make_wrangler(tree, trav, 8, exclude_self=True, precision="mixed")
    errs = []
    for f in (1e-30, 1.0, 1e30):
        qd = w64.reorder_sources(torch.as_tensor(q * f, device=cuda_device))
        mp = w64.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes,
                                 [qd])
        mp = w64.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                    trav.source_parent_boxes, mp)
        args = (None, trav.level_start_target_or_target_parent_box_nrs,
                trav.target_or_target_parent_boxes, trav.from_sep_siblings_starts,
                trav.from_sep_siblings_lists, mp)
        l64 = w64.multipole_to_local(*args)
        ltc = wtc.multipole_to_local(*args)
        wtc.check_status()
        errs.append(relerr(ltc.cpu(), l64.cpu()))
    assert max(errs) < 2e-6 and max(errs) < 1.5 * errs[1] + 1e-9, errs


@pytest.mark.parametrize("fmt", ["f16", "tf32"])
@pytest.mark.parametrize("geom", list(GEOMS))
@pytest.mark.parametrize("order", [4, 10])
def test_tensor_core_m2m_l2l_match_fp64(cuda_device, geom, order, fmt):
    """Mixed form with the tensor-core octant maps switched on: M2M and L2L
    as per-octant 3xTF32 GEMMs against the FP64 form on the same inputs."""
    src, tgt, tree, trav, tcls, q = _setup(geom)
    excl = tgt is None
    w64 = make_wrangler(tree, trav, order, exclude_self=excl)
    wtc = make_wrangler(tree, trav, order, exclude_self=excl, precision="mixed")
    assert wtc._tc_translations
    wtc.tc_m2m = wtc.tc_l2l = True
    wtc.tc_format = fmt
    qd = w64.reorder_sources(torch.as_tensor(q, device=cuda_device))
    mp = w64.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
    m64 = w64.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                 trav.source_parent_boxes, mp.clone())
    mtc = wtc.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                 trav.source_parent_boxes, mp.clone())
    wtc.check_status()
    assert relerr(mtc.cpu(), m64.cpu()) < 1e-6
    loc = w64.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                 trav.target_or_target_parent_boxes,
                                 trav.from_sep_siblings_starts, trav.from_sep_siblings_lists,
                                 m64)
    args = (None, trav.level_start_target_or_target_parent_box_nrs,
            trav.target_or_target_parent_boxes)
    l64 = w64.refine_locals(*args, loc.clone())
    ltc = wtc.refine_locals(*args, loc.clone())
    wtc.check_status()
    assert relerr(ltc.cpu(), l64.cpu()) < 1e-6
