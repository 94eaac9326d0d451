"""Adjoint FMM: the FMM on the transposed traversal is the exact transpose of
the forward FMM (dot-product identity, on the oracle and on the GPU), and
the autograd gradients (strengths, source and target positions) match the
FP64 direct-sum gradients and central finite differences."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sumpy_b200.adjoint import transpose_traversal
from sumpy_b200.tree import build_all
from tests._pointsets import sphere_plummer
from tests.test_tree import coverage_violations


def _separate():
    rng = np.random.default_rng(5)
    src = sphere_plummer(3000, 11)
    tgt = rng.standard_normal((3, 1200)) * 0.6
    return src, tgt


@pytest.mark.parametrize("case", ["separate", "self"])
def test_transposed_traversal_is_exact_transpose(case):
    src, tgt = _separate()
    if case == "self":
        tgt = None
    tree, trav, tcls = build_all(src, tgt, 12)
    tree_t, trav_t, tcls_t = transpose_traversal(tree, trav, tcls)
    assert coverage_violations(tree_t, trav_t) == 0
    rng = np.random.default_rng(2)
    q = rng.standard_normal(tree.nsources)
    g = rng.standard_normal(tree.ntargets)
    excl = case == "self"
    for p in (3, 6):
        fq = O.run_fmm(tree, trav, tcls, p, q, exclude_self=excl)
        ftg = O.run_fmm(tree_t, trav_t, tcls_t, p, g, exclude_self=excl)
        lhs, rhs = float(fq @ g), float(q @ ftg)
        scale = float(np.abs(fq).sum() * np.abs(g).max())
        assert abs(lhs - rhs) < 1e-13 * scale, (p, lhs, rhs)


def _shell_problem(ns=4000, nt=1500, seed=3):
    """Sphere sources perturbed radially, targets in the shell 2 <= r <= 3
    (the differentiable-potential workload, scaled down)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((3, ns))
    src = (1 + 0.05 * rng.standard_normal(ns)) * g / np.linalg.norm(g, axis=0)
    d = rng.standard_normal((3, nt))
    d /= np.linalg.norm(d, axis=0)
    tgt = np.cbrt(8 + 19 * rng.random(nt)) * d
    q = rng.standard_normal(ns)
    return src, tgt, q


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
@pytest.mark.parametrize("self_eval", [False, True])
def test_gpu_adjoint_dot_product(cuda_device, precision, tol, self_eval):
    from sumpy_b200.autograd import LaplaceFMM
    src, tgt, q = _shell_problem()
    if self_eval:
        src = sphere_plummer(4000, 9)
        tgt = None
    fmm = LaplaceFMM(order=6, max_particles_in_box=16, precision=precision, device=cuda_device)
    qt = torch.as_tensor(q, device=cuda_device).requires_grad_(True)
    phi = fmm(qt, torch.as_tensor(src, device=cuda_device),
              None if tgt is None else torch.as_tensor(tgt, device=cuda_device))
    g = torch.as_tensor(np.random.default_rng(8).standard_normal(phi.shape[0]), device=cuda_device)
    (phi * g).sum().backward()
    lhs = float((phi.detach() * g).sum())
    rhs = float((qt.detach() * qt.grad).sum())
    scale = float(phi.detach().abs().sum() * g.abs().max())
    assert abs(lhs - rhs) < tol * scale, (lhs, rhs)


def _direct_grads(src, tgt, q, g, dev):
    """FP64 direct-sum gradients of L with dL/dphi = g."""
    from sumpy_b200 import P2P, LaplaceKernel
    knl = [LaplaceKernel(3)]
    psi = P2P(knl, gradient=True)(None, src, tgt, (g,), device=dev)
    phi = P2P(knl, gradient=True)(None, tgt, src, (q,), device=dev)
    gq = psi[0]
    gsrc = torch.as_tensor(q, device=dev) * torch.stack(psi[1:4])
    gtgt = torch.as_tensor(g, device=dev) * torch.stack(phi[1:4])
    return gq, gsrc, gtgt


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_gradients_match_direct_sum(cuda_device, precision):
    from sumpy_b200 import P2P, LaplaceKernel
    from sumpy_b200.autograd import LaplaceFMM
    dev = cuda_device
    src, tgt, q = _shell_problem()
    # reference potential at unperturbed (radius 1) source positions
    src0 = src / np.linalg.norm(src, axis=0)
    (phi_ref,) = P2P([LaplaceKernel(3)])(None, tgt, src0, (q,), device=dev)
    fmm = LaplaceFMM(order=8, max_particles_in_box=32, precision=precision, device=dev)
    qt = torch.as_tensor(q, device=dev).requires_grad_(True)
    st = torch.as_tensor(src, device=dev).requires_grad_(True)
    tt = torch.as_tensor(tgt, device=dev).requires_grad_(True)
    phi = fmm(qt, st, tt)
    loss = 0.5 * ((phi - phi_ref) ** 2).sum()
    loss.backward()
    g = (phi - phi_ref).detach().cpu().numpy()
    gq, gsrc, gtgt = _direct_grads(src, tgt, q, g, dev)
    rel = lambda a, b: float((a - b).norm() / b.norm())
    assert rel(qt.grad, gq) < 1e-5
    # position gradients differentiate an order-8 expansion, which is one
    # order less accurate than its values: ~2e-5 at the sources (dense, small
    # boxes), ~2.5e-4 at the targets, which sit few to a box in the coarse
    # boxes of the shell; test_gpu_gradient_stages_are_exact_derivatives shows
    # the gradient kernels themselves are exact derivatives
    assert rel(st.grad, gsrc) < 5e-5
    assert rel(tt.grad, gtgt) < 1e-3


@pytest.mark.gpu
def test_gpu_gradients_match_finite_differences(cuda_device):
    """Central differences (h = 1e-4, FP64) on random strength and
    source-position coordinates.

    (a) The FMM loss 0.5*|F q - phi_ref|^2 is quadratic in q and the backward
        is the exact transpose, so its strength gradient matches FD of that
        same loss to rounding.
    (b) Seeded with the exact residual dL/dphi = phi_direct - phi_ref, the
        backward matches FD of the exact (direct-sum) loss to the FMM's
        truncation error, for strengths and source positions.
    """
    from sumpy_b200 import P2P, LaplaceKernel
    from sumpy_b200.autograd import LaplaceFMM
    dev = cuda_device
    src, tgt, q = _shell_problem(ns=2000, nt=800)
    src0 = src / np.linalg.norm(src, axis=0)
    knl = [LaplaceKernel(3)]
    (phi_ref,) = P2P(knl)(None, tgt, src0, (q,), device=dev)
    tgt_t = torch.as_tensor(tgt, device=dev)
    fmm = LaplaceFMM(order=8, max_particles_in_box=32, device=dev)
    rng = np.random.default_rng(4)
    h = 1e-4

    # (a) FD of the FMM loss with respect to strengths
    def loss_fmm(qq):
        phi = fmm(torch.as_tensor(qq, device=dev), torch.as_tensor(src, device=dev), tgt_t)
        return 0.5 * float(((phi - phi_ref) ** 2).sum())

    qt = torch.as_tensor(q, device=dev).requires_grad_(True)
    phi = fmm(qt, torch.as_tensor(src, device=dev), tgt_t)
    (0.5 * ((phi - phi_ref) ** 2).sum()).backward()
    for i in rng.choice(len(q), 6, replace=False):
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        fd = (loss_fmm(qp) - loss_fmm(qm)) / (2 * h)
        assert abs(fd - float(qt.grad[i])) < 1e-7 * max(abs(fd), 1.0), (i, fd, float(qt.grad[i]))

    # (b) exact residual through the backward, against FD of the exact loss
    def loss_direct(qq, ss):
        (p,) = P2P(knl)(None, tgt, ss, (qq,), device=dev)
        return 0.5 * float(((p - phi_ref) ** 2).sum())

    (phi_d,) = P2P(knl)(None, tgt, src, (q,), device=dev)
    qt = torch.as_tensor(q, device=dev).requires_grad_(True)
    st = torch.as_tensor(src, device=dev).requires_grad_(True)
    phi = fmm(qt, st, tgt_t)
    phi.backward(phi_d - phi_ref)
    errs_q, errs_x = [], []
    gq_scale = float(qt.grad.abs().max())
    for i in rng.choice(len(q), 8, replace=False):
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        fd = (loss_direct(qp, src) - loss_direct(qm, src)) / (2 * h)
        errs_q.append(abs(fd - float(qt.grad[i])) / gq_scale)
    gx_scale = float(st.grad.abs().max())
    for i in rng.choice(len(q), 8, replace=False):
        d = int(rng.integers(3))
        sp, sm = src.copy(), src.copy()
        sp[d, i] += h
        sm[d, i] -= h
        fd = (loss_direct(q, sp) - loss_direct(q, sm)) / (2 * h)
        errs_x.append(abs(fd - float(st.grad[d, i])) / gx_scale)
    assert max(errs_q) < 1e-5, errs_q
    assert max(errs_x) < 1e-4, errs_x


@pytest.mark.gpu
@pytest.mark.parametrize("stage", ["direct", "locals", "multipoles"])
def test_gpu_gradient_stages_are_exact_derivatives(cuda_device, stage):
    """With the tree fixed, the gradient form of each evaluation stage equals
    the central difference of that stage's values at shifted targets."""
    import dataclasses
    from tests.test_gpu_fmm import make_wrangler
    src, tgt = _separate()
    tree, trav, tcls = build_all(src, tgt, 12)
    q = torch.as_tensor(np.random.default_rng(1).standard_normal(tree.nsources),
                        device=cuda_device)

    def run(tr, gradient):
        tr._translation_classes = tcls
        w = make_wrangler(tr, dataclasses.replace(trav, tree=tr), 7)
        w.gradient = gradient
        qd = w.reorder_sources(q)
        if stage == "direct":
            return w.eval_direct(None, trav.target_boxes, trav.neighbor_source_boxes_starts,
                                 trav.neighbor_source_boxes_lists, [qd])
        mp = w.form_multipoles(None, trav.level_start_source_box_nrs, trav.source_boxes, [qd])
        mp = w.coarsen_multipoles(None, trav.level_start_source_parent_box_nrs,
                                  trav.source_parent_boxes, mp)
        if stage == "multipoles":
            return w.eval_multipoles(None, trav.target_boxes_sep_smaller_by_source_level,
                                     trav.from_sep_smaller_by_level, mp)
        loc = w.multipole_to_local(None, trav.level_start_target_or_target_parent_box_nrs,
                                   trav.target_or_target_parent_boxes,
                                   trav.from_sep_siblings_starts, trav.from_sep_siblings_lists, mp)
        loc = w.refine_locals(None, trav.level_start_target_or_target_parent_box_nrs,
                              trav.target_or_target_parent_boxes, loc)
        return w.eval_locals(None, trav.level_start_target_box_nrs, trav.target_boxes, loc)

    out = run(tree, True)
    h = 1e-5
    for d in range(3):
        tp, tm = tree.targets.copy(), tree.targets.copy()
        tp[d] += h
        tm[d] -= h
        vp = run(dataclasses.replace(tree, targets=tp), False)[0]
        vm = run(dataclasses.replace(tree, targets=tm), False)[0]
        fd = (vp - vm) / (2 * h)
        g = out[1 + d]
        assert float(g.abs().max()) > 0
        assert float((g - fd).abs().max() / g.abs().max()) < 1e-6, (stage, d)


# {{{ Helmholtz (complex strengths)

@pytest.mark.parametrize("case", ["separate", "self"])
def test_helmholtz_transposed_traversal_is_exact_transpose(case):
    """<F q, g> = <q, F^T g> (bilinear) on the Helmholtz oracle, k = 10."""
    src, tgt = _separate()
    if case == "self":
        tgt = None
    tree, trav, tcls = build_all(src, tgt, 12)
    tree_t, trav_t, tcls_t = transpose_traversal(tree, trav, tcls)
    rng = np.random.default_rng(4)
    q = rng.standard_normal(tree.nsources) + 1j * rng.standard_normal(tree.nsources)
    g = rng.standard_normal(tree.ntargets) + 1j * rng.standard_normal(tree.ntargets)
    excl = case == "self"
    for p in (3, 6):
        fq = O.run_fmm(tree, trav, tcls, p, q, exclude_self=excl, helmholtz_k=10.0)
        ftg = O.run_fmm(tree_t, trav_t, tcls_t, p, g, exclude_self=excl, helmholtz_k=10.0)
        lhs, rhs = complex(fq @ g), complex(q @ ftg)
        scale = float(np.abs(fq).sum() * np.abs(g).max())
        assert abs(lhs - rhs) < 1e-13 * scale, (p, lhs, rhs)


def fmm_direct(knl, tp, src, q, tts, k):
    from sumpy_b200 import P2P
    return P2P(knl, exclude_self=tts is not None)(None, tp, src, (q,), target_to_source=tts,
                                                  k=k)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("self_eval", [False, True])
def test_gpu_helmholtz_strength_gradient(cuda_device, self_eval):
    """q.grad of L = 0.5 |phi - phi_ref|^2 (PyTorch's complex convention:
    dL/dRe q + i dL/dIm q) against the direct-sum adjoint F^H (phi - phi_ref)
    and against central differences of the FMM itself."""
    from sumpy_b200 import P2P, HelmholtzKernel
    from sumpy_b200.autograd import HelmholtzFMM
    src, tgt, _ = _shell_problem(3000, 1200)
    rng = np.random.default_rng(8)
    q0 = rng.standard_normal(src.shape[1]) + 1j * rng.standard_normal(src.shape[1])
    k = 6.0
    fmm = HelmholtzFMM(order=12, k=k, precision="fp64", device=cuda_device)
    s = torch.as_tensor(src, device=cuda_device)
    t = None if self_eval else torch.as_tensor(tgt, device=cuda_device)
    tp = src if self_eval else tgt
    knl = [HelmholtzKernel(3)]
    tts = np.arange(src.shape[1]) if self_eval else None
    (phi_ref,) = P2P(knl, exclude_self=self_eval)(None, tp, src, (0.5 * q0,),
                                                   target_to_source=tts, k=k)

    def loss(qv):
        phi = fmm(qv, s, t)
        return 0.5 * ((phi - phi_ref).abs() ** 2).sum(), phi

    q = torch.as_tensor(q0, device=cuda_device).requires_grad_(True)
    L, phi = loss(q)
    L.backward()
    g = (phi - phi_ref).detach()
    # F^H g = conj(F^T conj(g)), F^T = the direct sum with the roles swapped
    (ftg,) = P2P(knl, exclude_self=self_eval)(None, src, tp, (g.conj().cpu().numpy(),),
                                              target_to_source=tts, k=k)
    ref = ftg.conj()
    err = float((q.grad - ref).norm() / ref.norm())
    # the same order's forward error against the direct sum bounds it
    fwd = float((phi.detach() - fmm_direct(knl, tp, src, q0, tts, k)).norm()
                / fmm_direct(knl, tp, src, q0, tts, k).norm())
    assert err < max(1e-5, 20 * fwd), (err, fwd)
    h = 1e-4
    for i in (0, 17, 1234):
        for unit in (1.0, 1j):
            qp = torch.as_tensor(q0, device=cuda_device).clone()
            qm = qp.clone()
            qp[i] += h * unit
            qm[i] -= h * unit
            fd = (float(loss(qp)[0]) - float(loss(qm)[0])) / (2 * h)
            an = float(q.grad[i].real if unit == 1.0 else q.grad[i].imag)
            assert abs(fd - an) < 1e-6 * max(abs(fd), 1.0), (i, unit, fd, an)

# }}}
