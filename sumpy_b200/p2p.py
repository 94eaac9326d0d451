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
