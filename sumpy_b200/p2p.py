"""All-pairs P2P (sumpy/p2p.py:215-285) on the GPU.

``P2P(target_kernels, exclude_self)(actx, targets, sources, (strength,))``
returns ``[potential]`` like sumpy's, computed by the FP64 CUDA kernel
``sumpy_p2p_direct_f64`` (``sumpy_helmholtz_p2p_direct_f64`` for a
``HelmholtzKernel``, whose wave number comes as a keyword argument, e.g.
``k=10``, as in sumpy). sumpy's FMM tests use this as the accuracy reference
(sumpy/test/test_fmm.py:284-286).
"""
from __future__ import annotations

import torch

from sumpy_b200 import _capi
from sumpy_b200._capi import call, dptr, stream_ptr
from sumpy_b200.kernel import HelmholtzKernel, helmholtz_k


def _soa(x, device):
    t = torch.as_tensor(x, dtype=torch.float64)
    if t.dim() != 2 or t.shape[0] != 3:
        raise ValueError("points must have shape (3, n)")
    return t.to(device).contiguous()


class P2P:
    """With ``gradient=True`` the call returns ``[potential, d/dx, d/dy, d/dz]``
    (derivatives with respect to the target coordinates)."""

    def __init__(self, target_kernels, exclude_self=False, strength_usage=None,
                 source_kernels=None, value_dtypes=None, name=None, gradient=False):
        if len(target_kernels) != 1:
            raise NotImplementedError("exactly one target kernel is supported")
        self.target_kernels = list(target_kernels)
        self.exclude_self = exclude_self
        self.gradient = gradient

    def __call__(self, actx, targets, sources, strength, target_to_source=None,
                 device="cuda", **kwargs):
        dev = torch.device(device)
        t = _soa(targets, dev)
        s = _soa(sources, dev)
        (q,) = strength
        knl = self.target_kernels[0]
        helm = isinstance(knl, HelmholtzKernel)
        if helm and self.gradient:
            raise NotImplementedError("gradient outputs are implemented for Laplace only")
        qdt = torch.complex128 if helm else torch.float64
        q = torch.as_tensor(q).to(dev, qdt).contiguous()
        tts = None
        if self.exclude_self:
            if target_to_source is None:
                raise ValueError("exclude_self needs target_to_source")
            tts = torch.as_tensor(target_to_source).to(dev, torch.int32).contiguous()
        scale = knl.global_scaling_const
        if helm:
            out = torch.empty(t.shape[1], dtype=torch.complex128, device=dev)
            call("sumpy_helmholtz_p2p_direct_f64", _capi.i64(t.shape[1]), dptr(t),
                 _capi.i64(t.shape[1]), _capi.i64(s.shape[1]), dptr(s), _capi.i64(s.shape[1]),
                 _capi.dbl(helmholtz_k(knl, kwargs)), dptr(q), dptr(tts), _capi.dbl(scale),
                 dptr(out), stream_ptr())
            return [out]
        args = (_capi.i64(t.shape[1]), dptr(t), _capi.i64(t.shape[1]), _capi.i64(s.shape[1]),
                dptr(s), _capi.i64(s.shape[1]), dptr(q), dptr(tts), _capi.dbl(scale))
        if self.gradient:
            buf = torch.empty((4, t.shape[1]), dtype=torch.float64, device=dev)
            call("sumpy_p2p_direct_grad_f64", *args, dptr(buf[0]), dptr(buf[1]), stream_ptr())
            return [buf[0], buf[1], buf[2], buf[3]]
        out = torch.empty(t.shape[1], dtype=torch.float64, device=dev)
        call("sumpy_p2p_direct_f64", *args, dptr(out), stream_ptr())
        return [out]


class _MatrixBase:
    def __init__(self, target_kernels, exclude_self=False, strength_usage=None,
                 source_kernels=None, value_dtypes=None, name=None):
        if len(target_kernels) != 1:
            raise NotImplementedError("exactly one target kernel is supported")
        self.target_kernels = list(target_kernels)
        self.exclude_self = exclude_self

    def _common(self, targets, sources, target_to_source, device, kwargs):
        dev = torch.device(device)
        t = _soa(targets, dev)
        s = _soa(sources, dev)
        tts = None
        if self.exclude_self:
            if target_to_source is None:
                raise ValueError("exclude_self needs target_to_source")
            tts = torch.as_tensor(target_to_source).to(dev, torch.int32).contiguous()
        knl = self.target_kernels[0]
        helm = isinstance(knl, HelmholtzKernel)
        k = helmholtz_k(knl, kwargs) if helm else None
        return dev, t, s, tts, knl.global_scaling_const, helm, k


class P2PMatrixGenerator(_MatrixBase):
    """The dense interaction matrix (sumpy/p2p.py:290-349):
    ``P2PMatrixGenerator(target_kernels, exclude_self)(actx, targets,
    sources, target_to_source=..., k=...)`` returns ``[M]`` with
    ``M[t, s] = scale * G(t - s)``, shape ``(ntargets, nsources)``, float64
    (complex128 for a ``HelmholtzKernel``); with ``exclude_self`` the
    entries with ``s == target_to_source[t]`` are 0. CUDA kernel
    ``sumpy_p2p_matrix_f64`` / ``sumpy_helmholtz_p2p_matrix_f64``."""

    def __call__(self, actx, targets, sources, target_to_source=None, device="cuda", **kwargs):
        dev, t, s, tts, scale, helm, k = self._common(targets, sources, target_to_source,
                                                      device, kwargs)
        nt, ns = t.shape[1], s.shape[1]
        out = torch.empty((nt, ns), dtype=torch.complex128 if helm else torch.float64,
                          device=dev)
        head = (_capi.i64(nt), dptr(t), _capi.i64(nt), _capi.i64(ns), dptr(s), _capi.i64(ns),
                dptr(tts))
        if helm:
            call("sumpy_helmholtz_p2p_matrix_f64", *head, _capi.dbl(k), _capi.dbl(scale),
                 dptr(out), stream_ptr())
        else:
            call("sumpy_p2p_matrix_f64", *head, _capi.dbl(scale), dptr(out), stream_ptr())
        return [out]


class P2PMatrixSubsetGenerator(_MatrixBase):
    """Entries of the interaction matrix at given index pairs
    (sumpy/p2p.py:354-477): ``P2PMatrixSubsetGenerator(target_kernels,
    exclude_self)(actx, targets, sources, tgtindices=..., srcindices=...,
    target_to_source=..., k=...)`` returns ``[r]`` with ``r[m] = scale *
    G(targets[:, tgtindices[m]] - sources[:, srcindices[m]])``. CUDA kernel
    ``sumpy_p2p_matrix_subset_f64`` / ``sumpy_helmholtz_p2p_matrix_subset_f64``."""

    def __call__(self, actx, targets, sources, *, tgtindices, srcindices,
                 target_to_source=None, device="cuda", **kwargs):
        dev, t, s, tts, scale, helm, k = self._common(targets, sources, target_to_source,
                                                      device, kwargs)
        ti = torch.as_tensor(tgtindices).to(dev)
        si = torch.as_tensor(srcindices).to(dev)
        if ti.shape != si.shape or ti.dim() != 1:
            raise ValueError("tgtindices and srcindices must be 1D arrays of the same size")
        # out-of-range indices would read outside the coordinate arrays
        if ti.numel():
            lim = torch.stack([ti.min().to(torch.int64), ti.max().to(torch.int64),
                               si.min().to(torch.int64), si.max().to(torch.int64)]).tolist()
            if lim[0] < 0 or lim[1] >= t.shape[1] or lim[2] < 0 or lim[3] >= s.shape[1]:
                raise IndexError("index out of range")
        ti = ti.to(torch.int32).contiguous()
        si = si.to(torch.int32).contiguous()
        n = ti.numel()
        out = torch.empty(n, dtype=torch.complex128 if helm else torch.float64, device=dev)
        head = (_capi.i64(n), dptr(ti), dptr(si), dptr(t), _capi.i64(t.shape[1]), dptr(s),
                _capi.i64(s.shape[1]), dptr(tts))
        if helm:
            call("sumpy_helmholtz_p2p_matrix_subset_f64", *head, _capi.dbl(k), _capi.dbl(scale),
                 dptr(out), stream_ptr())
        else:
            call("sumpy_p2p_matrix_subset_f64", *head, _capi.dbl(scale), dptr(out),
                 stream_ptr())
        return [out]
