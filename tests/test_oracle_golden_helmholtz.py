"""The Helmholtz oracle (oracle/helmholtz_oracle.c) against golden vectors
produced by sumpy's own HelmholtzKernel(3) expansion code at k = 5/2
(tests/golden/make_golden.py): P2M, P2L, L2P, M2P, M2M, L2L and M2L at
orders 2-4, the coefficient orderings, and the direct sum."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "helmholtz3d_operators.json")
DATA = json.load(open(GOLDEN))
CASES = DATA["cases"]
K = DATA["k"]
TOL = 1e-13


def cplx(v):
    a = np.asarray(v, dtype=float)
    return a[..., 0] + 1j * a[..., 1]


def rel(a, b):
    a = np.atleast_1d(np.asarray(a, dtype=complex))
    b = np.atleast_1d(np.asarray(b, dtype=complex))
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"p{c['order']}")
def test_coefficient_orderings(case):
    p = case["order"]
    assert O.stored_ids(p).tolist() == case["stored_ids"]
    assert O.full_ids(p).tolist() == case["full_ids"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"p{c['order']}")
def test_point_operators(case):
    p = case["order"]
    rs, rt = case["rscale_src"], case["rscale_tgt"]
    cin = np.array(case["coeffs_in"], dtype=complex)
    zero = np.zeros((3, 1))
    g = {k: cplx(case[k]["out"]) for k in
         ("p2m", "p2l", "l2p", "m2p", "m2m", "l2l", "m2l", "m2l_ratio")}
    assert rel(O.helm_p2m(p, rs, K, case["p2m"]["avec"], zero, [1.0]), g["p2m"]) < TOL
    assert rel(O.helm_p2l(p, rs, K, case["p2l"]["avec"], zero, [1.0]), g["p2l"]) < TOL
    assert rel(O.helm_l2p(p, rs, K, cin, case["l2p"]["bvec"]), g["l2p"]) < TOL
    assert rel(O.helm_m2p(p, rs, K, cin, case["m2p"]["bvec"]), g["m2p"]) < TOL
    assert rel(O.helm_m2m(p, p, rs, rt, K, case["m2m"]["dvec"], cin), g["m2m"]) < TOL
    assert rel(O.helm_l2l(p, p, rt, rs, K, case["l2l"]["dvec"], cin), g["l2l"]) < TOL
    assert rel(O.helm_m2l(p, rs, rs, K, case["m2l"]["dvec"], cin), g["m2l"]) < TOL
    assert rel(O.helm_m2l(p, rs, rt, K, case["m2l_ratio"]["dvec"], cin), g["m2l_ratio"]) < TOL


def test_k_zero_is_laplace():
    """At k = 0 every Helmholtz operator reduces to the Laplace one."""
    rng = np.random.default_rng(1)
    p, rs, rt = 4, 0.3, 0.6
    cin = rng.standard_normal((p + 1) ** 2)
    d = np.array([1.2, -0.7, 1.9])
    assert rel(O.helm_m2l(p, rs, rt, 0.0, d, cin), O.m2l(p, rs, rt, d, cin)) < 1e-13
    assert rel(O.helm_m2m(p, p, rs, rt, 0.0, d / 8, cin), O.m2m(p, p, rs, rt, d / 8, cin)) < 1e-13
    assert rel(O.helm_l2l(p, p, rt, rs, 0.0, d / 8, cin), O.l2l(p, p, rt, rs, d / 8, cin)) < 1e-13
    src = rng.uniform(-0.1, 0.1, (3, 5))
    q = rng.standard_normal(5)
    assert rel(O.helm_p2m(p, rs, 0.0, [0, 0, 0], src, q), O.p2m(p, rs, [0, 0, 0], src, q)) < 1e-13


def test_direct_sum():
    rng = np.random.default_rng(2)
    s = rng.random((3, 40))
    t = rng.random((3, 7)) + 2.0
    q = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    got = O.helm_p2p_direct(t, s, K, q)
    r = np.linalg.norm(t[:, :, None] - s[:, None, :], axis=0)
    ref = (q[None, :] * np.exp(1j * K * r) / r).sum(axis=1) / (4 * np.pi)
    assert rel(got, ref) < 1e-14


def test_oracle_detects_planted_error():
    case = CASES[-1]
    p = case["order"]
    cin = np.array(case["coeffs_in"], dtype=complex)
    out = O.helm_m2l(p, case["rscale_src"], case["rscale_src"], K, case["m2l"]["dvec"], cin)
    out[len(out) // 2] *= 1 + 1e-9
    assert rel(out, cplx(case["m2l"]["out"])) > TOL
