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
    assert rel(st.grad, gsrc) < 1e-5
    assert rel(tt.grad, gtgt) < 1e-5


@pytest.mark.gpu
def test_gpu_gradients_match_finite_differences(cuda_device):
    """Central differences (h = 1e-4, FP64) of the direct-sum loss on random
    strength and source-position coordinates."""
    from sumpy_b200 import P2P, LaplaceKernel
    from sumpy_b200.autograd import LaplaceFMM
    dev = cuda_device
    src, tgt, q = _shell_problem(ns=2000, nt=800)
    src0 = src / np.linalg.norm(src, axis=0)
    knl = [LaplaceKernel(3)]
    (phi_ref,) = P2P(knl)(None, tgt, src0, (q,), device=dev)
    phi_ref = phi_ref.cpu().numpy()

    def loss_direct(qq, ss):
        (phi,) = P2P(knl)(None, tgt, ss, (qq,), device=dev)
        return 0.5 * float(((phi.cpu().numpy() - phi_ref) ** 2).sum())

    fmm = LaplaceFMM(order=8, max_particles_in_box=32, device=dev)
    qt = torch.as_tensor(q, device=dev).requires_grad_(True)
    st = torch.as_tensor(src, device=dev).requires_grad_(True)
    phi = fmm(qt, st, torch.as_tensor(tgt, device=dev))
    (0.5 * ((phi - torch.as_tensor(phi_ref, device=dev)) ** 2).sum()).backward()
    rng = np.random.default_rng(4)
    h = 1e-4
    errs = []
    for i in rng.choice(len(q), 8, replace=False):
        qp, qm = q.copy(), q.copy()
        qp[i] += h
        qm[i] -= h
        fd = (loss_direct(qp, src) - loss_direct(qm, src)) / (2 * h)
        errs.append(abs(fd - float(qt.grad[i])) / max(abs(fd), 1e-30))
    gscale = float(st.grad.abs().max())
    for i in rng.choice(len(q), 8, replace=False):
        d = int(rng.integers(3))
        sp, sm = src.copy(), src.copy()
        sp[d, i] += h
        sm[d, i] -= h
        fd = (loss_direct(q, sp) - loss_direct(q, sm)) / (2 * h)
        errs.append(abs(fd - float(st.grad[d, i])) / gscale)
    assert max(errs) < 1e-4, errs
