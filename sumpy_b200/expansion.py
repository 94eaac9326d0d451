"""Expansion descriptors and host-side translation tables.

Mirrors the parts of sumpy's expansion classes the FMM path needs:
``LinearPDEConformingVolumeTaylorMultipoleExpansion`` and
``LinearPDEConformingVolumeTaylorLocalExpansion`` (sumpy/expansion/
multipole.py:416-419, local.py:512-515) -- their coefficient identifiers
and lengths -- plus the dense per-class M2L operators the CUDA GEMM applies.

Coefficient sets (3D Laplace and Helmholtz, sumpy/expansion/__init__.py:563-886):
the full set is every multi-index with |mi| <= p sorted by (|mi|, mi0, mi1, mi2);
the stored set keeps mi0 < 2, (p+1)^2 of them, in the same order. The
projection that restores the others is u_mi = -u_{mi-2e0+2e1} -
u_{mi-2e0+2e2} - k^2 rscale^2 u_{mi-2e0} (k = 0 for Laplace).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from functools import lru_cache
from typing import Any

import numpy as np

from sumpy_b200.kernel import HelmholtzKernel, LaplaceKernel


# {{{ index sets

@lru_cache(maxsize=None)
def full_ids(p: int) -> tuple:
    return tuple((i, j, deg - i - j)
                 for deg in range(p + 1)
                 for i in range(deg + 1)
                 for j in range(deg - i + 1))


@lru_cache(maxsize=None)
def stored_ids(p: int) -> tuple:
    return tuple(mi for mi in full_ids(p) if mi[0] < 2)


def stored_index(i, j, k):
    deg = i + j + k
    return deg * deg + i * (deg + 1) + j

# }}}


# {{{ expansion classes

@dataclass(frozen=True)
class _VolumeTaylorBase:
    kernel: Any
    order: int
    use_rscale: bool | None = None

    def __post_init__(self):
        if not isinstance(self.kernel, (LaplaceKernel, HelmholtzKernel)):
            raise NotImplementedError(
                "only LaplaceKernel(3) and HelmholtzKernel(3) expansions are implemented")
        if not 0 <= self.order <= 16:
            raise ValueError(f"order must be in [0, 16], got {self.order}")
        if self.use_rscale is False:
            raise NotImplementedError("expansions are always rscale-scaled")

    @property
    def dim(self):
        return 3

    def get_coefficient_identifiers(self):
        return list(stored_ids(self.order))

    def get_full_coefficient_identifiers(self):
        return list(full_ids(self.order))

    def __len__(self):
        return (self.order + 1) ** 2


@dataclass(frozen=True)
class LinearPDEConformingVolumeTaylorMultipoleExpansion(_VolumeTaylorBase):
    """Compressed Taylor multipole expansion (sumpy/expansion/multipole.py:416)."""


@dataclass(frozen=True)
class LinearPDEConformingVolumeTaylorLocalExpansion(_VolumeTaylorBase):
    """Compressed Taylor local expansion (sumpy/expansion/local.py:512).
    ``m2l_translation_override`` is accepted for call compatibility; the B200
    path always applies M2L as dense per-class operators."""
    m2l_translation_override: Any = field(default=None, compare=False)


@dataclass(frozen=True)
class VolumeTaylorLocalExpansion(_VolumeTaylorBase):
    """Uncompressed Taylor local expansion (sumpy/expansion/local.py:512-
    540): every mi with |mi| <= order. Used here by the QBX layer potential,
    whose value it determines through sum_{|mi| <= p} D^mi G(a) b^mi / mi!."""

    def get_coefficient_identifiers(self):
        return list(full_ids(self.order))

    def __len__(self):
        return (self.order + 1) * (self.order + 2) * (self.order + 3) // 6


@dataclass(frozen=True)
class LineTaylorLocalExpansion:
    """Taylor expansion along the line from the expansion center to one
    target (sumpy/expansion/local.py:116-185): coefficients
    d^i/dtau^i G(a + tau b) at tau = 0, i <= order, evaluated as their sum
    with 1/i!. Only meaningful where the target is known when coefficients
    are formed: the QBX layer potential (:mod:`sumpy_b200.qbx`)."""
    kernel: Any
    order: int
    use_rscale: bool | None = None

    def __post_init__(self):
        if not isinstance(self.kernel.get_base_kernel(), (LaplaceKernel, HelmholtzKernel)):
            raise NotImplementedError(
                "only LaplaceKernel(3) and HelmholtzKernel(3) expansions are implemented")
        if not 0 <= self.order <= 32:
            raise ValueError(f"order must be in [0, 32], got {self.order}")

    @property
    def dim(self):
        return 3

    def get_coefficient_identifiers(self):
        return [(i,) for i in range(self.order + 1)]

    def __len__(self):
        return self.order + 1

# }}}


# {{{ Laplace derivatives and M2L operators

def laplace_derivatives(vecs, rscale, maxdeg, maxi0=1):
    """Scaled derivatives ``rscale^|mi| d^mi (1/|x|)`` at points ``vecs``
    (shape (3, m)) for mi0 <= maxi0, |mi| <= maxdeg. Returns an array
    ``D[i, j, k, m]`` (entries with i + j + k > maxdeg are zero).

    Same recurrence as ``LaplaceDerivativeTaker.diff``
    (sumpy/derivative_taker.py:211-262), vectorised over points.
    """
    x = np.asarray(vecs, dtype=np.float64)
    m = x.shape[1]
    R = float(rscale)
    r2 = (x * x).sum(axis=0)
    r = np.sqrt(r2)
    xs = x / R
    rs2 = r2 / (R * R)
    M = maxdeg
    D = np.zeros((maxi0 + 1, M + 1, M + 1, m))

    def get(i, j, k):
        if i < 0 or j < 0 or k < 0:
            return 0.0
        return D[i, j, k]

    for deg in range(M + 1):
        for i in range(min(maxi0, deg) + 1):
            for j in range(deg - i + 1):
                k = deg - i - j
                mi = (i, j, k)
                if max(mi) <= 1:
                    if deg == 0:
                        v = 1.0 / r
                    elif deg == 1:
                        v = -x[mi.index(1)] / (r2 * r) * R
                    elif deg == 2:
                        a, b = [ax for ax in range(3) if mi[ax] == 1]
                        v = 3.0 * x[a] * x[b] / (r2 * r2 * r) * R * R
                    else:
                        v = -15.0 * x[0] * x[1] * x[2] / (r2 ** 3 * r) * R ** 3
                    D[i, j, k] = v
                    continue
                d = next(ax for ax in range(3) if mi[ax] >= 2)
                e = np.zeros(m)
                for ax in range(3):
                    n = mi[ax]
                    m1 = list(mi); m1[ax] -= 1
                    m2 = list(mi); m2[ax] -= 2
                    if ax == d:
                        e = e - (2 * n - 1) * xs[ax] * get(*m1) - (n - 1) ** 2 * get(*m2)
                    else:
                        e = e - 2 * n * xs[ax] * get(*m1) - n * (n - 1) * get(*m2)
                D[i, j, k] = e / rs2
    return D


def m2l_class_matrices(order, vectors, src_rscale, tgt_rscale):
    """Dense M2L operators T[c, t, s] for translation vectors ``vectors``
    (shape (3, nclasses), target center - source center).

    T[c, t, s] = (tgt_rscale/src_rscale)^|t| * D_c[s + t], with
    D_c = src_rscale^|mi| d^mi G(vector_c): the map sumpy applies per class
    (translation_classes_dependent_data, preprocess, Toeplitz product and
    postprocess; sumpy/expansion/m2l.py:363-389, 461-537, 539-558, 679-698).
    Derivatives with mi0 = 2 follow from the Laplace projection.
    """
    p = order
    ids = np.array(stored_ids(p))
    n = len(ids)
    D = laplace_derivatives(vectors, src_rscale, 2 * p, maxi0=1)
    nc = D.shape[-1]
    M = 2 * p
    # extend to mi0 == 2 via u_(2,j,k) = -u_(0,j+2,k) - u_(0,j,k+2)
    full = np.zeros((3, M + 3, M + 3, nc))
    full[:2, :M + 1, :M + 1] = D
    full[2, :M + 1, :M + 1] = -full[0, 2:M + 3, :M + 1] - full[0, :M + 1, 2:M + 3]
    s_plus_t = ids[None, :, :] + ids[:, None, :]          # [t, s, 3]
    T = full[s_plus_t[..., 0], s_plus_t[..., 1], s_plus_t[..., 2]]  # [t, s, nc]
    ratio = tgt_rscale / src_rscale
    deg_t = ids.sum(axis=1)
    T = T * (ratio ** deg_t)[:, None, None]
    return np.ascontiguousarray(np.moveaxis(T, -1, 0))   # [c, t, s]

# }}}


# {{{ Helmholtz derivatives and M2L operators

def helmholtz_derivatives(vecs, rscale, k, maxdeg, maxi0=1):
    """Scaled derivatives ``rscale^|mi| d^mi (exp(i k r)/r)`` at points
    ``vecs`` (shape (3, m)) for mi0 <= maxi0, |mi| <= maxdeg, as a complex
    array ``D[i, j, l, m]``.

    The recursion of ``RadialDerivativeTaker.diff`` with the Helmholtz base
    functions of ``HelmholtzDerivativeTaker.diff``
    (sumpy/derivative_taker.py:296-389), vectorised over points: with
    g_q = ((1/r) d/dr)^q G, D(mi, q) = x_a rs D(mi - e_a, q + 1) for the first
    axis a with mi_a == 1, else (mi_a - 1) rs^2 D(mi - 2e_a, q + 1) +
    x_a rs D(mi - e_a, q + 1) for the first axis with mi_a >= 2;
    D(0, q) = g_q, g_0 = e^{ikr}/r, g_1 = (ikr - 1) e^{ikr}/r^3,
    g_q = (-(2q - 1) g_{q-1} - k^2 g_{q-2}) / r^2.
    """
    x = np.asarray(vecs, dtype=np.float64)
    m = x.shape[1]
    rs = float(rscale)
    r2 = (x * x).sum(axis=0)
    r = np.sqrt(r2)
    eikr = np.exp(1j * k * r)
    M = maxdeg
    E = {}
    g = []
    for q in range(M + 1):
        if q == 0:
            v = eikr / r
        elif q == 1:
            v = (1j * k * r - 1.0) * eikr / (r2 * r)
        else:
            v = (-(2 * q - 1) * g[q - 1] - k * k * g[q - 2]) / r2
        g.append(v)
        E[(0, 0, 0, q)] = v
    for deg in range(1, M + 1):
        for i in range(min(maxi0, deg) + 1):
            for j in range(deg - i + 1):
                l = deg - i - j
                mi = (i, j, l)
                if 1 in mi:
                    ax, two = mi.index(1), False
                else:
                    ax, two = next(a for a in range(3) if mi[a] >= 2), True
                m1 = list(mi); m1[ax] -= 1
                m2 = list(mi); m2[ax] -= 2
                for q in range(M - deg + 1):
                    v = x[ax] * rs * E[(*m1, q + 1)]
                    if two:
                        v = v + (mi[ax] - 1) * rs * rs * E[(*m2, q + 1)]
                    E[(i, j, l, q)] = v
    D = np.zeros((maxi0 + 1, M + 1, M + 1, m), dtype=np.complex128)
    for (i, j, l, q), v in E.items():
        if q == 0:
            D[i, j, l] = v
    return D


def helmholtz_m2l_class_matrices(order, vectors, src_rscale, tgt_rscale, k):
    """Complex dense M2L operators T[c, t, s] of the Helmholtz kernel: as
    :func:`m2l_class_matrices`, with derivatives of exp(i k r)/r and the
    mi0 = 2 entries from the Helmholtz projection
    u_(2,j,l) = -u_(0,j+2,l) - u_(0,j,l+2) - k^2 src_rscale^2 u_(0,j,l)
    (get_full_kernel_derivatives_from_stored at the source rscale,
    sumpy/expansion/m2l.py:501-523)."""
    p = order
    ids = np.array(stored_ids(p))
    D = helmholtz_derivatives(vectors, src_rscale, k, 2 * p, maxi0=1)
    nc = D.shape[-1]
    M = 2 * p
    kappa = (k * src_rscale) ** 2
    full = np.zeros((3, M + 3, M + 3, nc), dtype=np.complex128)
    full[:2, :M + 1, :M + 1] = D
    full[2, :M + 1, :M + 1] = (-full[0, 2:M + 3, :M + 1] - full[0, :M + 1, 2:M + 3]
                               - kappa * full[0, :M + 1, :M + 1])
    s_plus_t = ids[None, :, :] + ids[:, None, :]
    T = full[s_plus_t[..., 0], s_plus_t[..., 1], s_plus_t[..., 2]]
    ratio = tgt_rscale / src_rscale
    T = T * (ratio ** ids.sum(axis=1))[:, None, None]
    return np.ascontiguousarray(np.moveaxis(T, -1, 0))


def real_embedding(T):
    """[c, t, s] complex -> [c, 2t + a, 2s + b] real with blocks
    [[Re, -Im], [Im, Re]]: applied to coefficient vectors stored as
    interleaved (re, im) pairs it is the complex product."""
    c, n, _ = T.shape
    R = np.empty((c, n, 2, n, 2))
    R[:, :, 0, :, 0] = T.real
    R[:, :, 0, :, 1] = -T.imag
    R[:, :, 1, :, 0] = T.imag
    R[:, :, 1, :, 1] = T.real
    return R.reshape(c, 2 * n, 2 * n)

# }}}


# {{{ M2M / L2L as dense per-octant operators

def _full_index_map(p):
    ids = full_ids(p)
    return {mi: f for f, mi in enumerate(ids)}, ids


def _shift_axis(V, p, ids, fidx, axis, dd, truncate_to=None):
    """Taylor shift of full coefficient columns V[full, cols] along one axis:
    multipole form out[mi] = sum_{q <= mi_a} V[mi with mi_a = q] dd^(mi_a - q)/(mi_a - q)!
    (truncate_to is None), local form out[mi] = sum_{q <= P - |mi|}
    V[mi + q e_a] dd^q / q! (truncate_to = P)."""
    from math import factorial
    out = np.zeros_like(V)
    for f, mi in enumerate(ids):
        if truncate_to is None:
            for q in range(mi[axis] + 1):
                m = list(mi); m[axis] = q
                out[f] += V[fidx[tuple(m)]] * dd ** (mi[axis] - q) / factorial(mi[axis] - q)
        else:
            deg = sum(mi)
            for q in range(truncate_to - deg + 1):
                m = list(mi); m[axis] += q
                out[f] += V[fidx[tuple(m)]] * dd ** q / factorial(q)
    return out


def _project(V, p, ids, fidx, kappa=0.0):
    """stored-embedded full columns -> full (the PDE projection, planes in order)."""
    V = V.copy()
    for f, mi in enumerate(ids):
        if mi[0] >= 2:
            i, j, k = mi
            V[f] = (-V[fidx[(i - 2, j + 2, k)]] - V[fidx[(i - 2, j, k + 2)]]
                    - kappa * V[fidx[(i - 2, j, k)]])
    return V


def _compress(V, p, ids, fidx, kappa=0.0):
    """full columns -> stored rows (transposed projection, rows in reverse)."""
    V = V.copy()
    for f in range(len(ids) - 1, -1, -1):
        i, j, k = ids[f]
        if i >= 2:
            V[fidx[(i - 2, j + 2, k)]] -= V[f]
            V[fidx[(i - 2, j, k + 2)]] -= V[f]
            V[fidx[(i - 2, j, k)]] -= kappa * V[f]
    return V[[fidx[mi] for mi in stored_ids(p)]]


def m2m_operator(order, src_rscale, tgt_rscale, dvec, kappa=0.0):
    """Dense M2M map [n_tgt, n_src] for one child -> parent offset
    ``dvec`` = parent center - child center: the child's stored coefficients
    in the parent's full slots times (r_src/r_tgt)^|mi|, shifted along axes
    1, 2, 0 by dvec/r_tgt, then compressed (sumpy/expansion/multipole.py:
    159-407). kappa = k^2 r_tgt^2 for Helmholtz."""
    p = order
    fidx, ids = _full_index_map(p)
    st = stored_ids(p)
    n = len(st)
    V = np.zeros((len(ids), n))
    ratio = src_rscale / tgt_rscale
    for s, mi in enumerate(st):
        V[fidx[mi], s] = ratio ** sum(mi)
    for axis in (1, 2, 0):
        V = _shift_axis(V, p, ids, fidx, axis, dvec[axis] / tgt_rscale)
    return _compress(V, p, ids, fidx, kappa)


def l2l_operator(order, src_rscale, tgt_rscale, dvec, kappa=0.0):
    """Dense L2L map [n_tgt, n_src] for one parent -> child offset ``dvec`` =
    child center - parent center: full derivatives from the stored ones
    (projection at r_src, kappa = k^2 r_src^2 for Helmholtz), truncated
    Taylor shift along axes 0, 1, 2 by dvec/r_src, times (r_tgt/r_src)^|mi|
    on the stored entries (sumpy/expansion/local.py:346-464)."""
    p = order
    fidx, ids = _full_index_map(p)
    st = stored_ids(p)
    n = len(st)
    V = np.zeros((len(ids), n))
    for s, mi in enumerate(st):
        V[fidx[mi], s] = 1.0
    V = _project(V, p, ids, fidx, kappa)
    for axis in (0, 1, 2):
        V = _shift_axis(V, p, ids, fidx, axis, dvec[axis] / src_rscale, truncate_to=p)
    ratio = tgt_rscale / src_rscale
    rows = np.array([fidx[mi] for mi in st])
    deg = np.array([sum(mi) for mi in st])
    return V[rows] * (ratio ** deg)[:, None]


def octant_offsets(h_child):
    """The 8 child-center offsets from the parent center, octant o = 4 bx + 2 by + bz
    (bit set = + side), for children of side h_child."""
    return np.array([[(1 if (o >> (2 - a)) & 1 else -1) * 0.5 * h_child for a in range(3)]
                     for o in range(8)])

# }}}
