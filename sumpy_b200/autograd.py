"""Differentiable 3D Laplace and Helmholtz FMMs: ``torch.autograd.Function``s
with hand-written backwards (:class:`LaplaceFMM`: strengths and positions;
:class:`HelmholtzFMM`: complex strengths).

``LaplaceFMM(order, ...)(strengths, sources, targets=None)`` returns the
potential phi(x_t) = sum_s q_s / (4 pi |x_t - x_s|) at the targets (at the
sources, self excluded, when ``targets`` is None). Gradients:

* strengths: F^T g, the FMM on the transposed traversal of the same tree
  (:func:`sumpy_b200.adjoint.transpose_traversal`);
* source positions: q_s * grad psi(x_s), psi = F^T g evaluated with the
  gradient forms of P2P/L2P/M2P (target-derivative kernels);
* target positions: g_t * grad phi(x_t) from the gradient form of the
  forward evaluation.

No expansion is kept between forward and backward: the backward builds its
own multipoles and locals (recomputation instead of storage).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from sumpy_b200.adjoint import transpose_traversal
from sumpy_b200.drive import drive_fmm
from sumpy_b200.expansion import (
    LinearPDEConformingVolumeTaylorLocalExpansion,
    LinearPDEConformingVolumeTaylorMultipoleExpansion,
)
from sumpy_b200.fmm import SumpyExpansionWrangler, SumpyTreeIndependentDataForWrangler
from sumpy_b200.kernel import HelmholtzKernel, LaplaceKernel
from sumpy_b200.tree import build_all


@dataclass(frozen=True)
class _Config:
    order: int
    max_particles_in_box: int
    precision: str
    device: torch.device


def _wrangler(cfg, tree, trav, tcls, exclude_self, gradient):
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: LinearPDEConformingVolumeTaylorMultipoleExpansion(knl, o),
        lambda o, **kw: LinearPDEConformingVolumeTaylorLocalExpansion(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: cfg.order,
                                  translation_classes_data=tcls, precision=cfg.precision,
                                  device=cfg.device, gradient=gradient)


class _FMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, strengths, sources, targets, cfg):
        self_eval = targets is None
        src = sources.detach().to("cpu", torch.float64).numpy()
        tgt = None if self_eval else targets.detach().to("cpu", torch.float64).numpy()
        tree, trav, tcls = build_all(src, tgt, cfg.max_particles_in_box)
        pos_grad = (sources.requires_grad if self_eval
                    else targets is not None and targets.requires_grad)
        w = _wrangler(cfg, tree, trav, tcls, self_eval, gradient=pos_grad)
        q = strengths.detach().to(cfg.device, torch.float64).contiguous()
        out = drive_fmm(None, w, [q])
        ctx.cfg = cfg
        ctx.self_eval = self_eval
        ctx.geometry = (tree, trav, tcls)
        ctx.grad_phi = torch.stack(out[1:4]) if pos_grad else None
        ctx.save_for_backward(q)
        return out[0]

    @staticmethod
    def backward(ctx, g):
        (q,) = ctx.saved_tensors
        cfg = ctx.cfg
        need_q, need_src, need_tgt = ctx.needs_input_grad[:3]
        tree_t, trav_t, tcls_t = transpose_traversal(*ctx.geometry)
        wa = _wrangler(cfg, tree_t, trav_t, tcls_t, ctx.self_eval, gradient=need_src)
        g = g.to(cfg.device, torch.float64).contiguous()
        out = drive_fmm(None, wa, [g])
        grad_q = out[0] if need_q else None
        grad_src = grad_tgt = None
        if need_src:
            grad_src = q * torch.stack(out[1:4])
            if ctx.self_eval:
                # each point is also a target: add g * grad phi
                grad_src = grad_src + g * ctx.grad_phi
        if need_tgt and not ctx.self_eval:
            grad_tgt = g * ctx.grad_phi
        return grad_q, grad_src, grad_tgt, None


class LaplaceFMM:
    """Callable differentiable FMM for the 3D Laplace potential.

    :arg order: expansion order (same on every level).
    :arg precision: ``"fp64"`` or ``"mixed"`` (see :class:`SumpyExpansionWrangler`).
    """

    def __init__(self, order=8, max_particles_in_box=32, precision="fp64", device="cuda"):
        self.cfg = _Config(int(order), int(max_particles_in_box), precision,
                           torch.device(device))

    def __call__(self, strengths, sources, targets=None):
        """strengths: (ns,), sources: (3, ns), targets: (3, nt) or None."""
        return _FMMFunction.apply(strengths, sources, targets, self.cfg)


@dataclass(frozen=True)
class _HConfig:
    order: int
    k: float
    max_particles_in_box: int
    precision: str
    device: torch.device


def _helm_wrangler(cfg, tree, trav, tcls, exclude_self):
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: LinearPDEConformingVolumeTaylorMultipoleExpansion(knl, o),
        lambda o, **kw: LinearPDEConformingVolumeTaylorLocalExpansion(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.complex128, lambda kn, a, t, lev: cfg.order,
                                  kernel_extra_kwargs={"k": cfg.k},
                                  translation_classes_data=tcls, precision=cfg.precision,
                                  device=cfg.device)


class _HelmholtzFunction(torch.autograd.Function):
    """phi = F q for complex strengths q. With PyTorch's convention for
    complex gradients, q.grad = F^H g = conj(F^T conj(g)); F^T is the FMM on
    the transposed traversal (G(x - y) = G(y - x) and D(-x) = S D(x) hold for
    every radial kernel, and the Helmholtz projection keeps the parity of
    |mi|, so the derivation in sumpy_b200.adjoint carries over)."""

    @staticmethod
    def forward(ctx, strengths, sources, targets, cfg):
        self_eval = targets is None
        src = sources.detach().to("cpu", torch.float64).numpy()
        tgt = None if self_eval else targets.detach().to("cpu", torch.float64).numpy()
        tree, trav, tcls = build_all(src, tgt, cfg.max_particles_in_box)
        w = _helm_wrangler(cfg, tree, trav, tcls, self_eval)
        q = strengths.detach().to(cfg.device, torch.complex128).contiguous()
        (phi,) = drive_fmm(None, w, [q])
        ctx.cfg = cfg
        ctx.self_eval = self_eval
        ctx.geometry = (tree, trav, tcls)
        return phi

    @staticmethod
    def backward(ctx, g):
        cfg = ctx.cfg
        if not ctx.needs_input_grad[0]:
            return None, None, None, None
        tree_t, trav_t, tcls_t = transpose_traversal(*ctx.geometry)
        wa = _helm_wrangler(cfg, tree_t, trav_t, tcls_t, ctx.self_eval)
        g = g.to(cfg.device, torch.complex128).conj().contiguous()
        (psi,) = drive_fmm(None, wa, [g])
        return psi.conj(), None, None, None


class HelmholtzFMM:
    """Callable FMM for the 3D Helmholtz potential
    phi(x_t) = sum_s q_s e^{ik|x_t - x_s|} / (4 pi |x_t - x_s|), differentiable
    with respect to the complex strengths (the adjoint FMM).

    :arg order: expansion order (same on every level).
    :arg k: real wave number.
    :arg precision: ``"fp64"`` or ``"mixed"``.
    """

    def __init__(self, order=14, k=1.0, max_particles_in_box=32, precision="fp64",
                 device="cuda"):
        self.cfg = _HConfig(int(order), float(k), int(max_particles_in_box), precision,
                            torch.device(device))

    def __call__(self, strengths, sources, targets=None):
        """strengths: (ns,) complex, sources: (3, ns), targets: (3, nt) or None."""
        return _HelmholtzFunction.apply(strengths, sources, targets, self.cfg)
