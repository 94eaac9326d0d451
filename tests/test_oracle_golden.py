"""The FP64 oracle against golden vectors produced by sumpy's own expansion
code (tests/golden/make_golden.py): P2M, P2L, L2P, M2P, M2M, L2L and M2L at
every order the file holds (2-6), plus the coefficient orderings."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "laplace3d_operators.json")
CASES = json.load(open(GOLDEN))["cases"]
TOL = 1e-13


def rel(a, b):
    a = np.atleast_1d(np.asarray(a, dtype=float))
    b = np.atleast_1d(np.asarray(b, dtype=float))
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"p{c['order']}")
def test_coefficient_orderings(case):
    p = case["order"]
    assert O.stored_ids(p).tolist() == case["stored_ids"]
    assert O.full_ids(p).tolist() == case["full_ids"]
    assert case["ncoeff"] == (p + 1) ** 2


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"p{c['order']}")
def test_point_operators(case):
    p = case["order"]
    rs, rt = case["rscale_src"], case["rscale_tgt"]
    cin = np.array(case["coeffs_in"])
    zero = np.zeros((3, 1))
    assert rel(O.p2m(p, rs, case["p2m"]["avec"], zero, [1.0]), case["p2m"]["out"]) < TOL
    assert rel(O.p2l(p, rs, case["p2l"]["avec"], zero, [1.0]), case["p2l"]["out"]) < TOL
    assert rel(O.l2p(p, rs, cin, case["l2p"]["bvec"]), case["l2p"]["out"]) < TOL
    assert rel(O.m2p(p, rs, cin, case["m2p"]["bvec"]), case["m2p"]["out"]) < TOL
    assert rel(O.m2m(p, p, rs, rt, case["m2m"]["dvec"], cin), case["m2m"]["out"]) < TOL
    assert rel(O.l2l(p, p, rt, rs, case["l2l"]["dvec"], cin), case["l2l"]["out"]) < TOL
    assert rel(O.m2l(p, rs, rs, case["m2l"]["dvec"], cin), case["m2l"]["out"]) < TOL
    assert rel(O.m2l(p, rs, rt, case["m2l_ratio"]["dvec"], cin), case["m2l_ratio"]["out"]) < TOL


def test_oracle_detects_planted_error():
    """A perturbed operator output must fail the golden comparison."""
    case = CASES[-1]
    p = case["order"]
    cin = np.array(case["coeffs_in"])
    out = O.m2l(p, case["rscale_src"], case["rscale_src"], case["m2l"]["dvec"], cin)
    out[len(out) // 2] *= 1 + 1e-9
    assert rel(out, case["m2l"]["out"]) > TOL
