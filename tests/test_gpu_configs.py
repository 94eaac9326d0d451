"""Parity at the benchmark configurations themselves (CUDA path against the
oracle or the FP64 direct sum, never against itself).

* 3D Laplace, 20,000 sources and 20,000 separate targets uniform in
  [0, 1]^3 (seeds 15 and 18), strengths N(0, 1) (seed 44), p = 6,
  max_particles_in_box 30: the FP64 form equals the oracle (sumpy's
  algorithm restated) to 1e-12 and the direct sum to the FMM's truncation
  error; the mixed form stays within 1e-6 of the oracle. This is the case of
  sumpy's test_sumpy_fmm / test_unified_single_and_double
  (sumpy/test/test_fmm.py:78-297, 386-469) at the benchmark's size.
* The 1M-point sphere + Plummer workload (sources = targets, exclude_self),
  p = 10 on the leaf-96 tree and p = 13 on the leaf-128 tree: relative L2
  error of the mixed and FP64 forms on 4,096 sampled targets against the
  FP64 direct sum, bounded at the measured values (p = 10: 3.46e-6 mixed,
  3.39e-6 FP64; p = 13: 9.6e-7 mixed, meeting relL2 <= 1e-6).
* 3D Helmholtz (k = 10), p = 14, sources = targets on the unit sphere, at
  20,000 points (the oracle's size): FP64 form against the oracle to 1e-11,
  mixed form within 1e-5 of it, both against the direct sum.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sumpy_b200 import (
    P2P,
    HelmholtzKernel,
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


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def wrangler(knl, trav, tcls, order, precision, dev, exclude_self, dtype=np.float64,
             extra=None):
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: MExp(knl, o), lambda o, **kw: LExp(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, dtype, lambda *a: order,
                                  kernel_extra_kwargs=extra or {},
                                  translation_classes_data=tcls, precision=precision,
                                  device=dev)


def test_uniform_20k_p6_matches_oracle_and_direct_sum(cuda_device):
    dev = cuda_device
    src = np.random.default_rng(15).random((3, 20_000))
    tgt = np.random.default_rng(18).random((3, 20_000))
    q = np.random.default_rng(44).standard_normal(20_000)
    tree, trav, tcls = build_all(src, tgt, 30)
    knl = LaplaceKernel(3)
    ref = O.run_fmm(tree, trav, tcls, 6, q)
    qd = torch.as_tensor(q, device=dev)
    (pot64,) = drive_fmm(None, wrangler(knl, trav, tcls, 6, "fp64", dev, False), [qd])
    wmx = wrangler(knl, trav, tcls, 6, "mixed", dev, False)
    (potmx,) = drive_fmm(None, wmx, [qd])
    wmx.check_status()
    (direct,) = P2P([knl])(None, tgt, src, (q,), device=dev)
    pot64, potmx, direct = pot64.cpu().numpy(), potmx.cpu().numpy(), direct.cpu().numpy()
    assert rel(pot64, ref) < 1e-12
    assert rel(potmx, ref) < 1e-6
    # truncation error of order 6 on this tree (measured 1.26e-4)
    e = rel(pot64, direct)
    assert 1e-6 < e < 2e-4, e
    assert abs(rel(potmx, direct) - e) < 1e-6


@pytest.fixture(scope="module")
def sphere_plummer_1m(cuda_device):
    dev = cuda_device
    pts = sphere_plummer(1_000_000, 2024)
    q = np.random.default_rng(44).standard_normal(1_000_000)
    sample = np.random.default_rng(99).choice(1_000_000, size=4096, replace=False)
    (ref,) = P2P([LaplaceKernel(3)], exclude_self=True)(
        None, pts[:, sample], pts, (q,), target_to_source=sample, device=dev)
    return pts, torch.as_tensor(q, device=dev), sample, ref.cpu().numpy()


@pytest.mark.parametrize("order,leaf,bound_mixed,bound_fp64", [
    (10, 96, 3.6e-6, 3.5e-6),
    (13, 128, 1.0e-6, 5.0e-7),
])
def test_sphere_plummer_1m_accuracy_against_direct_sum(cuda_device, sphere_plummer_1m, order,
                                                       leaf, bound_mixed, bound_fp64):
    dev = cuda_device
    pts, qd, sample, ref = sphere_plummer_1m
    tree, trav, tcls = build_all(pts, None, leaf)
    knl = LaplaceKernel(3)
    errs = {}
    pots = {}
    for precision in ("mixed", "fp64"):
        w = wrangler(knl, trav, tcls, order, precision, dev, True)
        (pot,) = drive_fmm(None, w, [qd])
        w.check_status()
        pots[precision] = pot.cpu().numpy()[sample]
        errs[precision] = rel(pots[precision], ref)
        del w
        torch.cuda.empty_cache()
    assert errs["mixed"] < bound_mixed, errs
    assert errs["fp64"] < bound_fp64, errs
    # the two forms agree far below the truncation error
    assert rel(pots["mixed"], pots["fp64"]) < 1e-6, errs


def test_helmholtz_sphere_p14_matches_oracle_and_direct_sum(cuda_device):
    dev = cuda_device
    k = 10.0
    rng = np.random.default_rng(2025)
    g = rng.standard_normal((3, 20_000))
    pts = g / np.linalg.norm(g, axis=0)
    q = rng.standard_normal(20_000) + 1j * rng.standard_normal(20_000)
    tree, trav, tcls = build_all(pts, None, 64)
    knl = HelmholtzKernel(3)
    ref = O.run_fmm(tree, trav, tcls, 14, q, exclude_self=True, helmholtz_k=k)
    qd = torch.as_tensor(q, device=dev)
    kw = dict(dtype=np.complex128, extra={"k": k})
    (pot64,) = drive_fmm(None, wrangler(knl, trav, tcls, 14, "fp64", dev, True, **kw), [qd])
    wmx = wrangler(knl, trav, tcls, 14, "mixed", dev, True, **kw)
    (potmx,) = drive_fmm(None, wmx, [qd])
    wmx.check_status()
    (direct,) = P2P([knl], exclude_self=True)(None, pts, pts, (q,),
                                              target_to_source=np.arange(20_000),
                                              device=dev, k=k)
    pot64, potmx, direct = pot64.cpu().numpy(), potmx.cpu().numpy(), direct.cpu().numpy()
    assert rel(pot64, ref) < 1e-11
    assert rel(potmx, ref) < 1e-5
    assert rel(pot64, direct) < 1e-5
    assert rel(potmx, direct) < 1e-5
