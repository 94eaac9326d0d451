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

Geometry cache. A :class:`LaplaceFMM` (or :class:`HelmholtzFMM`) object keeps
the tree, traversal, translation classes, the transposed traversal and the
wranglers built on them (each replaying its evaluation from a CUDA graph)
from one call to the next. A call whose points all lie inside the boxes they
were sorted into reuses them and only overwrites the device coordinates
(:meth:`SumpyExpansionWrangler.set_positions`); a point that left its box, a
change of size, or ``rebuild=True`` builds the geometry anew. With the boxes
fixed, the FMM is a smooth function of the positions and the position
gradients are the exact derivatives of the values the forward returns, so
central differences of the forward agree with the backward to the
differences' own truncation error.
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
    cuda_graph: bool = True


def _wrangler(cfg, tree, trav, tcls, exclude_self, gradient):
    knl = LaplaceKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: LinearPDEConformingVolumeTaylorMultipoleExpansion(knl, o),
        lambda o, **kw: LinearPDEConformingVolumeTaylorLocalExpansion(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.float64, lambda k, a, t, lev: cfg.order,
                                  translation_classes_data=tcls, precision=cfg.precision,
                                  device=cfg.device, gradient=gradient,
                                  cuda_graph=cfg.cuda_graph)


def _owner(starts, counts_nonchild, n):
    """Box owning each particle in tree order (particles of a box that are
    not in its children, boxtree's ``*_counts_nonchild``)."""
    starts = np.asarray(starts, dtype=np.int64)
    cnt = np.asarray(counts_nonchild, dtype=np.int64)
    boxes = np.nonzero(cnt)[0]
    out = np.full(n, -1, dtype=np.int64)
    for_box = np.repeat(boxes, cnt[boxes])
    first = np.cumsum(cnt[boxes]) - cnt[boxes]
    pos = np.repeat(starts[boxes] - first, cnt[boxes]) + np.arange(int(cnt[boxes].sum()))
    out[pos] = for_box
    if (out < 0).any():
        raise ValueError("tree leaves a particle without an owning box")
    return out


class _Geometry:
    """Tree, traversal, translation classes, their transpose, and the
    wranglers on them, for one set of source (and target) positions; reused
    while every point stays inside its box (closed box, as the tree sorted
    it)."""

    def __init__(self, cfg, src, tgt, make_wrangler):
        self.cfg = cfg
        self.self_eval = tgt is None
        if cfg.device.type == "cuda":
            # the tree is built on the GPU from the device coordinates
            s = src.detach().to(cfg.device, torch.float64)
            t = None if self.self_eval else tgt.detach().to(cfg.device, torch.float64)
            self.tree, self.trav, self.tcls = build_all(s, t, cfg.max_particles_in_box,
                                                        device=cfg.device)
        else:
            s = src.detach().to("cpu", torch.float64).numpy()
            t = None if self.self_eval else tgt.detach().to("cpu", torch.float64).numpy()
            self.tree, self.trav, self.tcls = build_all(s, t, cfg.max_particles_in_box)
        self._transposed = None
        self._make = make_wrangler
        self._fwd = {}
        self._bwd = {}
        tree = self.tree
        dev = cfg.device
        # closed boxes, widened by a rounding margin of the key computation
        half = (0.5 * tree.root_extent * np.exp2(-np.asarray(tree.box_levels, np.float64))
                + 1e-12 * tree.root_extent)
        lo = np.asarray(tree.box_centers) - half
        hi = np.asarray(tree.box_centers) + half
        so = _owner(tree.box_source_starts, tree.box_source_counts_nonchild, tree.nsources)
        self.src_perm = torch.as_tensor(np.asarray(tree.user_source_ids, np.int64), device=dev)
        self.src_lo = torch.as_tensor(lo[:, so], device=dev)
        self.src_hi = torch.as_tensor(hi[:, so], device=dev)
        if self.self_eval:
            self.tgt_perm = self.tgt_lo = self.tgt_hi = None
        else:
            to = _owner(tree.box_target_starts, tree.box_target_counts_nonchild, tree.ntargets)
            inv = np.empty(tree.ntargets, dtype=np.int64)
            inv[np.asarray(tree.sorted_target_ids, np.int64)] = np.arange(tree.ntargets)
            self.tgt_perm = torch.as_tensor(inv, device=dev)
            self.tgt_lo = torch.as_tensor(lo[:, to], device=dev)
            self.tgt_hi = torch.as_tensor(hi[:, to], device=dev)
        self.src_sorted = None
        self.tgt_sorted = None
        self.version = 0

    def sorted_positions(self, src, tgt):
        """(sources, targets) in tree order on the device, or None when a
        point lies outside its box or the sizes differ."""
        dev = self.cfg.device
        if (tgt is None) != self.self_eval or src.shape[-1] != self.tree.nsources:
            return None
        if tgt is not None and tgt.shape[-1] != self.tree.ntargets:
            return None
        s = src.detach().to(dev, torch.float64)[:, self.src_perm].contiguous()
        inside = ((s >= self.src_lo) & (s <= self.src_hi)).all()
        t = None
        if tgt is not None:
            t = tgt.detach().to(dev, torch.float64)[:, self.tgt_perm].contiguous()
            inside = inside & ((t >= self.tgt_lo) & (t <= self.tgt_hi)).all()
        if not bool(inside):
            return None
        return s, t

    def set_positions(self, s, t):
        """Tree-order coordinates into every wrangler built so far."""
        self.src_sorted, self.tgt_sorted = s, t
        tt = s if t is None else t
        for w in self._fwd.values():
            w.set_positions(s, tt)
        for w in self._bwd.values():
            w.set_positions(tt, s)
        self.version += 1

    def transposed(self):
        if self._transposed is None:
            self._transposed = transpose_traversal(self.tree, self.trav, self.tcls)
        return self._transposed

    def forward_wrangler(self, gradient=False):
        w = self._fwd.get(gradient)
        if w is None:
            w = self._make(self.cfg, self.tree, self.trav, self.tcls, self.self_eval, gradient)
            if self.src_sorted is not None:
                w.set_positions(self.src_sorted,
                                self.src_sorted if self.tgt_sorted is None else self.tgt_sorted)
            self._fwd[gradient] = w
        return w

    def backward_wrangler(self, gradient=False):
        w = self._bwd.get(gradient)
        if w is None:
            tree_t, trav_t, tcls_t = self.transposed()
            w = self._make(self.cfg, tree_t, trav_t, tcls_t, self.self_eval, gradient)
            if self.src_sorted is not None:
                w.set_positions(self.src_sorted if self.tgt_sorted is None else self.tgt_sorted,
                                self.src_sorted)
            self._bwd[gradient] = w
        return w


class _GeometryCache:
    """The geometry of the last call and the counters of reuse."""

    def __init__(self, make_wrangler):
        self.make = make_wrangler
        self.geo = None
        self.builds = 0
        self.reuses = 0

    def get(self, cfg, src, tgt, rebuild=False):
        geo = self.geo
        pos = None
        if geo is not None and not rebuild and geo.cfg == cfg:
            pos = geo.sorted_positions(src, tgt)
        if pos is None:
            self.geo = geo = _Geometry(cfg, src, tgt, self.make)
            pos = geo.sorted_positions(src, tgt)
            if pos is None:
                raise RuntimeError("a freshly built tree does not contain its own points")
            self.builds += 1
        else:
            self.reuses += 1
        geo.set_positions(*pos)
        return geo


class _FMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, strengths, sources, targets, cfg, cache, rebuild):
        self_eval = targets is None
        geo = cache.get(cfg, sources, targets, rebuild)
        pos_grad = (sources.requires_grad if self_eval
                    else targets is not None and targets.requires_grad)
        w = geo.forward_wrangler(gradient=pos_grad)
        q = strengths.detach().to(cfg.device, torch.float64).contiguous()
        out = drive_fmm(None, w, [q])
        ctx.cfg = cfg
        ctx.self_eval = self_eval
        ctx.geo = geo
        ctx.version = geo.version
        ctx.positions = (geo.src_sorted, geo.tgt_sorted)
        ctx.grad_phi = torch.stack(out[1:4]) if pos_grad else None
        ctx.save_for_backward(q)
        return out[0]

    @staticmethod
    def backward(ctx, g):
        (q,) = ctx.saved_tensors
        cfg = ctx.cfg
        need_q, need_src, need_tgt = ctx.needs_input_grad[:3]
        geo = ctx.geo
        if geo.version != ctx.version:
            # a later call moved the points of this geometry: restore this call's
            geo.set_positions(*ctx.positions)
        grad_q = grad_src = grad_tgt = None
        if need_q or need_src:
            wa = geo.backward_wrangler(gradient=need_src)
            g = g.to(cfg.device, torch.float64).contiguous()
            out = drive_fmm(None, wa, [g])
            grad_q = out[0] if need_q else None
            if need_src:
                grad_src = q * torch.stack(out[1:4])
                if ctx.self_eval:
                    # each point is also a target: add g * grad phi
                    grad_src = grad_src + g * ctx.grad_phi
        if need_tgt and not ctx.self_eval:
            grad_tgt = g.to(cfg.device, torch.float64) * ctx.grad_phi
        return grad_q, grad_src, grad_tgt, None, None, None


class LaplaceFMM:
    """Callable differentiable FMM for the 3D Laplace potential.

    :arg order: expansion order (same on every level).
    :arg precision: ``"fp64"`` or ``"mixed"`` (see :class:`SumpyExpansionWrangler`).
    :arg cuda_graph: replay each evaluation from a CUDA graph (captured on
        the first evaluation of a geometry).

    The object keeps its last geometry (see the module docstring); the
    counters ``geometry_builds`` and ``geometry_reuses`` say how often it
    was built and reused.
    """

    def __init__(self, order=8, max_particles_in_box=32, precision="fp64", device="cuda",
                 cuda_graph=True):
        self.cfg = _Config(int(order), int(max_particles_in_box), precision,
                           torch.device(device), bool(cuda_graph))
        self._cache = _GeometryCache(_wrangler)

    @property
    def geometry_builds(self):
        return self._cache.builds

    @property
    def geometry_reuses(self):
        return self._cache.reuses

    def __call__(self, strengths, sources, targets=None, rebuild=False):
        """strengths: (ns,), sources: (3, ns), targets: (3, nt) or None;
        ``rebuild``: build the tree anew even if the points fit the old one."""
        return _FMMFunction.apply(strengths, sources, targets, self.cfg, self._cache,
                                  bool(rebuild))


@dataclass(frozen=True)
class _HConfig:
    order: int
    k: float
    max_particles_in_box: int
    precision: str
    device: torch.device
    cuda_graph: bool = True


def _helm_wrangler(cfg, tree, trav, tcls, exclude_self, gradient=False):
    if gradient:
        raise NotImplementedError("Helmholtz position gradients are not implemented")
    knl = HelmholtzKernel(3)
    ti = SumpyTreeIndependentDataForWrangler(
        None, lambda o, **kw: LinearPDEConformingVolumeTaylorMultipoleExpansion(knl, o),
        lambda o, **kw: LinearPDEConformingVolumeTaylorLocalExpansion(knl, o), [knl],
        exclude_self=exclude_self)
    return SumpyExpansionWrangler(ti, trav, np.complex128, lambda kn, a, t, lev: cfg.order,
                                  kernel_extra_kwargs={"k": cfg.k},
                                  translation_classes_data=tcls, precision=cfg.precision,
                                  device=cfg.device, cuda_graph=cfg.cuda_graph)


class _HelmholtzFunction(torch.autograd.Function):
    """phi = F q for complex strengths q. With PyTorch's convention for
    complex gradients, q.grad = F^H g = conj(F^T conj(g)); F^T is the FMM on
    the transposed traversal (G(x - y) = G(y - x) and D(-x) = S D(x) hold for
    every radial kernel, and the Helmholtz projection keeps the parity of
    |mi|, so the derivation in sumpy_b200.adjoint carries over)."""

    @staticmethod
    def forward(ctx, strengths, sources, targets, cfg, cache, rebuild):
        if sources.requires_grad or (targets is not None and targets.requires_grad):
            raise NotImplementedError("HelmholtzFMM differentiates with respect to the "
                                      "strengths only")
        geo = cache.get(cfg, sources, targets, rebuild)
        w = geo.forward_wrangler()
        q = strengths.detach().to(cfg.device, torch.complex128).contiguous()
        (phi,) = drive_fmm(None, w, [q])
        ctx.cfg = cfg
        ctx.geo = geo
        ctx.version = geo.version
        ctx.positions = (geo.src_sorted, geo.tgt_sorted)
        return phi

    @staticmethod
    def backward(ctx, g):
        cfg = ctx.cfg
        if not ctx.needs_input_grad[0]:
            return None, None, None, None, None, None
        geo = ctx.geo
        if geo.version != ctx.version:
            geo.set_positions(*ctx.positions)
        wa = geo.backward_wrangler()
        g = g.to(cfg.device, torch.complex128).conj().contiguous()
        (psi,) = drive_fmm(None, wa, [g])
        return psi.conj(), None, None, None, None, None


class HelmholtzFMM:
    """Callable FMM for the 3D Helmholtz potential
    phi(x_t) = sum_s q_s e^{ik|x_t - x_s|} / (4 pi |x_t - x_s|), differentiable
    with respect to the complex strengths (the adjoint FMM).

    :arg order: expansion order (same on every level).
    :arg k: real wave number.
    :arg precision: ``"fp64"`` or ``"mixed"``.

    Keeps its last geometry like :class:`LaplaceFMM`.
    """

    def __init__(self, order=14, k=1.0, max_particles_in_box=32, precision="fp64",
                 device="cuda", cuda_graph=True):
        self.cfg = _HConfig(int(order), float(k), int(max_particles_in_box), precision,
                            torch.device(device), bool(cuda_graph))
        self._cache = _GeometryCache(_helm_wrangler)

    @property
    def geometry_builds(self):
        return self._cache.builds

    @property
    def geometry_reuses(self):
        return self._cache.reuses

    def __call__(self, strengths, sources, targets=None, rebuild=False):
        """strengths: (ns,) complex, sources: (3, ns), targets: (3, nt) or None."""
        return _HelmholtzFunction.apply(strengths, sources, targets, self.cfg, self._cache,
                                        bool(rebuild))
