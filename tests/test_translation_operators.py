"""Host-built dense translation maps (the per-octant M2M/L2L operators the
tensor-core M2M applies, and the M2L class operators) against the oracles'
restatement of sumpy's translations, Laplace and Helmholtz."""
import numpy as np
import pytest

from oracle import oracle as O
from sumpy_b200.expansion import (
    helmholtz_m2l_class_matrices,
    l2l_operator,
    m2l_class_matrices,
    m2m_operator,
    octant_offsets,
)


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize("order", [2, 5, 10])
def test_octant_operators_laplace(order):
    rng = np.random.default_rng(order)
    rp, rc = 0.4, 0.2
    offs = octant_offsets(0.25)
    c = rng.standard_normal((order + 1) ** 2)
    for o in range(8):
        d = offs[o]
        assert rel(m2m_operator(order, rc, rp, -d) @ c, O.m2m(order, order, rc, rp, -d, c)) < 1e-13
        assert rel(l2l_operator(order, rp, rc, d) @ c, O.l2l(order, order, rp, rc, d, c)) < 1e-13


@pytest.mark.parametrize("order", [3, 8])
def test_octant_operators_helmholtz(order):
    rng = np.random.default_rng(order)
    rp, rc, k = 0.4, 0.2, 7.0
    offs = octant_offsets(0.25)
    c = rng.standard_normal((order + 1) ** 2) + 1j * rng.standard_normal((order + 1) ** 2)
    for o in (0, 3, 7):
        d = offs[o]
        m = m2m_operator(order, rc, rp, -d, (k * rp) ** 2) @ c
        assert rel(m, O.helm_m2m(order, order, rc, rp, k, -d, c)) < 1e-13
        l = l2l_operator(order, rp, rc, d, (k * rp) ** 2) @ c
        assert rel(l, O.helm_l2l(order, order, rp, rc, k, d, c)) < 1e-13


def test_m2l_class_operators():
    rng = np.random.default_rng(0)
    d = np.array([[1.25], [-0.625], [1.875]])
    for p in (4, 9):
        c = rng.standard_normal((p + 1) ** 2)
        T = m2l_class_matrices(p, d, 0.3, 0.3)[0]
        assert rel(T @ c, O.m2l(p, 0.3, 0.3, d[:, 0], c)) < 1e-13
        cz = c + 1j * rng.standard_normal((p + 1) ** 2)
        T = helmholtz_m2l_class_matrices(p, d, 0.3, 0.6, 4.0)[0]
        assert rel(T @ cz, O.helm_m2l(p, 0.3, 0.6, 4.0, d[:, 0], cz)) < 1e-13
