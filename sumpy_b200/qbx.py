"""QBX layer potentials with sumpy's interface (sumpy/qbx.py:84-420).

:class:`LayerPotential` evaluates, for every target t with its expansion
center c_t, the local expansion about c_t of every source, summed with the
source strengths (quadrature weights and area elements folded in, as in
sumpy, qbx.py:305-310); :class:`LayerPotentialMatrixGenerator` writes the
matrix of those pair values and :class:`LayerPotentialMatrixSubsetGenerator`
selected entries of it. All three run the CUDA kernels behind
``sumpy_qbx_*`` (``sumpy_b200/csrc/qbx.cu``) in FP64 (complex128 for
Helmholtz) and return torch CUDA tensors.

Expansions: :class:`~sumpy_b200.expansion.LineTaylorLocalExpansion`,
:class:`~sumpy_b200.expansion.VolumeTaylorLocalExpansion` and
:class:`~sumpy_b200.expansion.LinearPDEConformingVolumeTaylorLocalExpansion`.
Their values coincide (the degree-i terms of a volume Taylor sum are the
i-th line Taylor term); they differ for target derivatives, which the line
form applies to each coefficient (d/da, a = center - source) and the volume
forms to the evaluated sum (d/db, b = target - center), as sumpy does
(qbx.py:121-137).

Kernels: LaplaceKernel(3) and HelmholtzKernel(3) (wave number by name in
the keyword arguments), optionally wrapped once in AxisTargetDerivative
(target side) or AxisSourceDerivative / DirectionalSourceDerivative
(source side; the direction vectors by name, shape (3, nsources)). A pair
of a target kernel and a source kernel carries at most one derivative.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from sumpy_b200._capi import call, dptr, stream_ptr
from sumpy_b200._lib import load_cuda_library
from sumpy_b200.expansion import (
    LinearPDEConformingVolumeTaylorLocalExpansion,
    LineTaylorLocalExpansion,
    VolumeTaylorLocalExpansion,
)
from sumpy_b200.kernel import (
    AxisSourceDerivative,
    AxisTargetDerivative,
    DirectionalSourceDerivative,
    HelmholtzKernel,
    LaplaceKernel,
    helmholtz_k,
)

_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double

# kernel modes of sumpy_qbx_* (sumpy_b200/csrc/qbx.cu)
MODE_VALUE = 0
MODE_TGT_DERIV_LINE = 1
MODE_TGT_DERIV_VOLUME = 2
MODE_SRC_DERIV_AXIS = 3
MODE_SRC_DERIV_DIR = 4


def _unwrap(kernel, target):
    """(base kernel, derivative descriptor or None) of a target or source
    kernel with at most one derivative wrapper."""
    if target and isinstance(kernel, AxisTargetDerivative):
        base, deriv = kernel.inner_kernel, ("tgt", kernel.axis)
    elif not target and isinstance(kernel, AxisSourceDerivative):
        base, deriv = kernel.inner_kernel, ("src", kernel.axis)
    elif not target and isinstance(kernel, DirectionalSourceDerivative):
        base, deriv = kernel.inner_kernel, ("dir", kernel.dir_vec_name)
    else:
        base, deriv = kernel, None
    if not isinstance(base, (LaplaceKernel, HelmholtzKernel)):
        raise NotImplementedError(
            f"QBX kernel {kernel}: one derivative of LaplaceKernel(3) / HelmholtzKernel(3)")
    return base, deriv


def _points(a, name, device):
    t = torch.as_tensor(a, dtype=torch.float64, device=device)
    if t.ndim != 2 or t.shape[0] != 3:
        raise ValueError(f"{name} must have shape (3, n); got {tuple(t.shape)}")
    return t.contiguous()


class LayerPotentialBase:
    """``sumpy.qbx.LayerPotentialBase`` (sumpy/qbx.py:84-246)."""

    def __init__(self, expansion, strength_usage=None, value_dtypes=None, name=None,
                 device=None, source_kernels=None, target_kernels=None):
        if not isinstance(expansion, (LineTaylorLocalExpansion, VolumeTaylorLocalExpansion,
                                      LinearPDEConformingVolumeTaylorLocalExpansion)):
            raise NotImplementedError(f"QBX expansion {type(expansion).__name__}")
        if target_kernels is None or source_kernels is None:
            raise TypeError("target_kernels and source_kernels must be given")
        self.expansion = expansion
        self.target_kernels = tuple(target_kernels)
        self.source_kernels = tuple(source_kernels)
        if strength_usage is None:
            strength_usage = list(range(len(self.source_kernels)))
        if len(strength_usage) != len(self.source_kernels):
            raise ValueError("one strength_usage entry per source kernel")
        self.strength_usage = tuple(strength_usage)
        self.strength_count = max(self.strength_usage) + 1 if self.strength_usage else 0
        self.name = name or self.default_name
        self.device = torch.device(device if device is not None else "cuda")
        bases = {_unwrap(k, True)[0] for k in self.target_kernels} | \
            {_unwrap(k, False)[0] for k in self.source_kernels}
        if len(bases) != 1:
            raise ValueError("all target and source kernels must share one base kernel")
        self.base_kernel = bases.pop()
        self.helmholtz = isinstance(self.base_kernel, HelmholtzKernel)
        self.value_dtypes = tuple(value_dtypes) if value_dtypes is not None else tuple(
            np.complex128 if self.helmholtz else np.float64 for _ in self.target_kernels)
        self.line = isinstance(expansion, LineTaylorLocalExpansion)

    default_name = "qbx"

    @property
    def nresults(self):
        return len(self.target_kernels)

    def _pair_mode(self, tknl, sknl, kwargs, sources):
        """(mode, axis, direction tensor) of one (target, source) kernel pair."""
        _, td = _unwrap(tknl, True)
        _, sd = _unwrap(sknl, False)
        if td is not None and sd is not None:
            raise NotImplementedError("a target and a source derivative together (second "
                                      "derivatives) are not implemented")
        if td is not None:
            return (MODE_TGT_DERIV_LINE if self.line else MODE_TGT_DERIV_VOLUME), td[1], None
        if sd is None:
            return MODE_VALUE, 0, None
        if sd[0] == "src":
            return MODE_SRC_DERIV_AXIS, sd[1], None
        if sd[1] not in kwargs:
            raise TypeError(f"the directional source derivative needs '{sd[1]}'")
        dirs = _points(kwargs[sd[1]], sd[1], self.device)
        if dirs.shape[1] != sources.shape[1]:
            raise ValueError(f"{sd[1]} needs one vector per source")
        return MODE_SRC_DERIV_DIR, 0, dirs

    def _k(self, kwargs):
        return helmholtz_k(self.base_kernel, kwargs) if self.helmholtz else 0.0

    def _geometry(self, targets, sources, centers):
        load_cuda_library()
        t = _points(targets, "targets", self.device)
        s = _points(sources, "sources", self.device)
        c = _points(centers, "centers", self.device)
        if c.shape[1] != t.shape[1]:
            raise ValueError("one expansion center per target")
        return t, s, c


class LayerPotential(LayerPotentialBase):
    """Direct applier for the layer potential (sumpy/qbx.py:250-340)."""

    default_name = "qbx_apply"

    def __call__(self, actx, targets, sources, centers, strengths, expansion_radii, **kwargs):
        """:arg strengths: one density per strength index, with area elements
        and quadrature weights already multiplied in. Returns one result per
        target kernel (torch CUDA tensors)."""
        t, s, c = self._geometry(targets, sources, centers)
        nt, ns = t.shape[1], s.shape[1]
        if len(strengths) < self.strength_count:
            raise ValueError(f"{self.strength_count} strength arrays needed")
        cdt = torch.complex128 if self.helmholtz else torch.float64
        dens = [torch.as_tensor(d, device=self.device).to(cdt).contiguous() for d in strengths]
        for d in dens:
            if d.shape != (ns,):
                raise ValueError("each strength array needs one entry per source")
        k = self._k(kwargs)
        out = []
        for tknl in self.target_kernels:
            res = torch.zeros(nt, dtype=cdt, device=self.device)
            for sknl, use in zip(self.source_kernels, self.strength_usage):
                mode, axis, dirs = self._pair_mode(tknl, sknl, kwargs, s)
                part = torch.empty(nt, dtype=cdt, device=self.device)
                args = [_i(self.expansion.order), _i(mode), _i(axis)]
                if self.helmholtz:
                    args.append(_d(k))
                args += [_i64(nt), dptr(t), _i64(nt), dptr(c), _i64(nt), _i64(ns), dptr(s),
                         _i64(ns), dptr(dirs), _i64(ns), dptr(dens[use]),
                         _d(self.base_kernel.global_scaling_const), dptr(part), stream_ptr()]
                call("sumpy_qbx_lpot_helmholtz_f64" if self.helmholtz
                     else "sumpy_qbx_lpot_laplace_f64", *args)
                res += part
            out.append(res)
        return tuple(out)


class LayerPotentialMatrixGenerator(LayerPotentialBase):
    """Layer potential matrix entries (sumpy/qbx.py:345-420): result[i] is
    the (ntargets, nsources) matrix of target kernel i, summed over the
    source kernels (unit strengths)."""

    default_name = "qbx_matrix"

    def __call__(self, actx, targets, sources, centers, expansion_radii, **kwargs):
        t, s, c = self._geometry(targets, sources, centers)
        nt, ns = t.shape[1], s.shape[1]
        cdt = torch.complex128 if self.helmholtz else torch.float64
        k = self._k(kwargs)
        out = []
        for tknl in self.target_kernels:
            mat = torch.zeros((nt, ns), dtype=cdt, device=self.device)
            for sknl in self.source_kernels:
                mode, axis, dirs = self._pair_mode(tknl, sknl, kwargs, s)
                part = torch.empty((nt, ns), dtype=cdt, device=self.device)
                args = [_i(self.expansion.order), _i(mode), _i(axis)]
                if self.helmholtz:
                    args.append(_d(k))
                args += [_i64(nt), dptr(t), _i64(nt), dptr(c), _i64(nt), _i64(ns), dptr(s),
                         _i64(ns), dptr(dirs), _i64(ns),
                         _d(self.base_kernel.global_scaling_const), dptr(part), stream_ptr()]
                call("sumpy_qbx_matrix_helmholtz_f64" if self.helmholtz
                     else "sumpy_qbx_matrix_laplace_f64", *args)
                mat += part
            out.append(mat)
        return tuple(out)


class LayerPotentialMatrixSubsetGenerator(LayerPotentialBase):
    """Selected layer potential matrix entries (sumpy/qbx.py:425-520):
    result[i][m] is entry (tgtindices[m], srcindices[m]) of target kernel i's
    matrix."""

    default_name = "qbx_subset"

    def __call__(self, actx, targets, sources, centers, expansion_radii, tgtindices,
                 srcindices, **kwargs):
        t, s, c = self._geometry(targets, sources, centers)
        ti = torch.as_tensor(tgtindices, device=self.device).to(torch.int32).contiguous()
        si = torch.as_tensor(srcindices, device=self.device).to(torch.int32).contiguous()
        if ti.shape != si.shape or ti.ndim != 1:
            raise ValueError("tgtindices and srcindices must be 1D arrays of one length")
        n = ti.numel()
        if n and (int(ti.min()) < 0 or int(ti.max()) >= t.shape[1] or int(si.min()) < 0
                  or int(si.max()) >= s.shape[1]):
            raise IndexError("matrix entry index out of range")
        cdt = torch.complex128 if self.helmholtz else torch.float64
        k = self._k(kwargs)
        nt, ns = t.shape[1], s.shape[1]
        out = []
        for tknl in self.target_kernels:
            vals = torch.zeros(n, dtype=cdt, device=self.device)
            for sknl in self.source_kernels:
                mode, axis, dirs = self._pair_mode(tknl, sknl, kwargs, s)
                part = torch.empty(n, dtype=cdt, device=self.device)
                args = [_i(self.expansion.order), _i(mode), _i(axis)]
                if self.helmholtz:
                    args.append(_d(k))
                args += [_i64(n), dptr(ti), dptr(si), dptr(t), _i64(nt), dptr(c), _i64(nt),
                         dptr(s), _i64(ns), dptr(dirs), _i64(ns),
                         _d(self.base_kernel.global_scaling_const), dptr(part), stream_ptr()]
                call("sumpy_qbx_matrix_subset_helmholtz_f64" if self.helmholtz
                     else "sumpy_qbx_matrix_subset_laplace_f64", *args)
                vals += part
            out.append(vals)
        return tuple(out)
