"""CPU oracle for QBX layer potentials (numpy, FP64).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by the CPU-baseline /
reference arm of ``bench.py``. The product package ``sumpy_b200`` never
imports it.

Restates the pair expression of sumpy's layer potential kernels
(sumpy/qbx.py:113-157, the loop bodies at qbx.py:279-292, 359-372, 468-478):
with a = center - source and b = target - center, a source contributes the
order-p local Taylor expansion of its kernel about the center, evaluated at
the target. For the line Taylor expansion (sumpy/expansion/local.py:116-185)
that is sum_{i <= p} c_i with c_i = (1/i!) d^i/dtau^i G(a + tau b) at tau = 0;
for the volume Taylor expansions (local.py:225-309) it is
sum_{|mi| <= p} D^mi G(a) b^mi / mi!, whose degree-i part is the same c_i.

Method (independent of the device kernels' recurrences): Taylor-mode
automatic differentiation. The series of G(a + tau b) in tau is built with
truncated power-series arithmetic (product, square root, reciprocal and
exponential of series, e.g. Griewank and Walther, "Evaluating Derivatives",
ch. 13) from |a + tau b|^2 = |a|^2 + 2 a.b tau + |b|^2 tau^2, every
coefficient being a dual number (value, derivative) seeded along the
direction a derivative is taken in:

* target derivative, line Taylor: d/da_axis of each coefficient (sumpy
  applies the target kernel's postprocess to the coefficients with avec,
  qbx.py:121-132, and AxisTargetDerivative differentiates by that vector,
  sumpy/kernel.py:2350-2371);
* target derivative, volume Taylor: d/db_axis of the truncated sum (the
  expansion's evaluate, local.py:284-309);
* AxisSourceDerivative: -d/da_axis (sumpy/kernel.py:2308-2318);
* DirectionalSourceDerivative: -dir . grad_a (sumpy/kernel.py:2466-2481).

Parity of this oracle is pinned to sumpy's own symbolic expansion code
through the golden pairs in ``tests/golden/qbx3d_pairs.json`` (written by
``tests/golden/make_golden.py --which qbx``).
"""
from __future__ import annotations

import numpy as np

VALUE, TGT_DERIV_LINE, TGT_DERIV_VOLUME, SRC_DERIV_AXIS, SRC_DERIV_DIR = range(5)


class _Dual:
    """Elementwise dual numbers v + eps d over numpy arrays (real or complex)."""

    __slots__ = ("v", "d")

    def __init__(self, v, d=None):
        self.v = v
        self.d = np.zeros_like(v) if d is None else d

    def __add__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v + o.v, self.d + o.d)
        return _Dual(self.v + o, self.d)

    __radd__ = __add__

    def __sub__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v - o.v, self.d - o.d)
        return _Dual(self.v - o, self.d)

    def __mul__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v * o.v, self.v * o.d + self.d * o.v)
        return _Dual(self.v * o, self.d * o)

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v / o.v, (self.d * o.v - self.v * o.d) / (o.v * o.v))
        return _Dual(self.v / o, self.d / o)


def _dsqrt(x):
    s = np.sqrt(x.v)
    return _Dual(s, x.d / (2.0 * s))


def _dexp(x):
    e = np.exp(x.v)
    return _Dual(e, x.d * e)


def _series_sqrt(q, p):
    r = [_dsqrt(q[0])]
    for n in range(1, p + 1):
        acc = q[n] if n < len(q) else _Dual(np.zeros_like(q[0].v))
        for i in range(1, n):
            acc = acc - r[i] * r[n - i]
        r.append(acc / (2.0 * r[0]))
    return r


def _series_recip(r, p):
    g = [_Dual(np.ones_like(r[0].v)) / r[0]]
    for n in range(1, p + 1):
        acc = r[1] * g[n - 1]
        for j in range(2, n + 1):
            acc = acc + r[j] * g[n - j]
        g.append(acc * (-1.0) / r[0])
    return g


def _series_exp(x, p):
    e = [_dexp(x[0])]
    for n in range(1, p + 1):
        acc = x[1] * e[n - 1] * 1.0
        for j in range(2, n + 1):
            acc = acc + x[j] * e[n - j] * float(j)
        e.append(acc / float(n))
    return e


def _series_mul(f, g, p):
    out = []
    for n in range(p + 1):
        acc = f[0] * g[n]
        for j in range(1, n + 1):
            acc = acc + f[j] * g[n - j]
        out.append(acc)
    return out


def line_coefficients(order, a, b, k=None, seed_a=None, seed_b=None):
    """Taylor coefficients c_0..c_order of G(a + tau b) in tau, as duals.

    a, b: arrays of shape (3, n). G = 1/|d| (Laplace) when k is None, else
    exp(i k |d|)/|d| (Helmholtz). seed_a / seed_b (shape (3, n) or None): the
    derivative direction of a / b carried in the dual parts."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    za = np.zeros_like(a) if seed_a is None else np.asarray(seed_a, float)
    zb = np.zeros_like(b) if seed_b is None else np.asarray(seed_b, float)
    A = _Dual(np.sum(a * a, 0), 2.0 * np.sum(a * za, 0))
    D = _Dual(np.sum(a * b, 0), np.sum(za * b + a * zb, 0))
    B = _Dual(np.sum(b * b, 0), 2.0 * np.sum(b * zb, 0))
    q = [A, D * 2.0, B]
    r = _series_sqrt(q, order)
    g = _series_recip(r, order)
    if k is None:
        return g
    ikr = [_Dual(1j * k * x.v, 1j * k * x.d) for x in r]
    return _series_mul(_series_exp(ikr, order), g, order)


def pair_values(order, mode, a, b, k=None, axis=0, dirs=None):
    """The QBX pair expression (kernel scaling not applied) for every column
    of a = center - source and b = target - center (shape (3, n))."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    n = a.shape[1]
    e = np.zeros((3, n))
    if mode in (TGT_DERIV_LINE, TGT_DERIV_VOLUME, SRC_DERIV_AXIS):
        e[axis] = 1.0
    elif mode == SRC_DERIV_DIR:
        e = np.asarray(dirs, float)
    seed_a = e if mode in (TGT_DERIV_LINE, SRC_DERIV_AXIS, SRC_DERIV_DIR) else None
    seed_b = e if mode == TGT_DERIV_VOLUME else None
    c = line_coefficients(order, a, b, k, seed_a, seed_b)
    tot = c[0]
    for x in c[1:]:
        tot = tot + x
    if mode == VALUE:
        return tot.v
    if mode in (TGT_DERIV_LINE, TGT_DERIV_VOLUME):
        return tot.d
    return -tot.d


def _pairs(targets, centers, sources, ti, si):
    t = np.asarray(targets, float)
    c = np.asarray(centers, float)
    s = np.asarray(sources, float)
    return c[:, ti] - s[:, si], t[:, ti] - c[:, ti]


def matrix(order, mode, targets, centers, sources, k=None, axis=0, dirs=None, scale=1.0):
    """(ntargets, nsources) matrix of scaled pair values."""
    nt = np.asarray(targets).shape[1]
    ns = np.asarray(sources).shape[1]
    ti, si = np.meshgrid(np.arange(nt), np.arange(ns), indexing="ij")
    ti, si = ti.ravel(), si.ravel()
    a, b = _pairs(targets, centers, sources, ti, si)
    d = None if dirs is None else np.asarray(dirs, float)[:, si]
    return scale * pair_values(order, mode, a, b, k, axis, d).reshape(nt, ns)


def matrix_subset(order, mode, targets, centers, sources, tgtindices, srcindices, k=None,
                  axis=0, dirs=None, scale=1.0):
    ti = np.asarray(tgtindices)
    si = np.asarray(srcindices)
    a, b = _pairs(targets, centers, sources, ti, si)
    d = None if dirs is None else np.asarray(dirs, float)[:, si]
    return scale * pair_values(order, mode, a, b, k, axis, d)


def lpot(order, mode, targets, centers, sources, strength, k=None, axis=0, dirs=None,
         scale=1.0, block=256):
    """Layer potential at each target: sum over sources of strength times
    the scaled pair value (blocked over targets to bound memory)."""
    nt = np.asarray(targets).shape[1]
    strength = np.asarray(strength)
    out = np.zeros(nt, dtype=np.complex128 if k is not None else np.float64)
    for t0 in range(0, nt, block):
        sl = slice(t0, min(nt, t0 + block))
        m = matrix(order, mode, np.asarray(targets)[:, sl], np.asarray(centers)[:, sl],
                   sources, k, axis, dirs, scale)
        out[sl] = m @ strength
    return out
