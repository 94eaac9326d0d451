"""The QBX oracle (oracle/qbx_oracle.py) against golden pair values from
sumpy's own expansion code (tests/golden/qbx3d_pairs.json, written by
tests/golden/make_golden.py --which qbx), against the closed-form layer
potentials of the unit sphere, and the host-side checks of
sumpy_b200.qbx (no GPU needed)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import qbx_oracle as q
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
)
from sumpy_b200.qbx import (
    LayerPotential,
    LayerPotentialMatrixGenerator,
    MODE_TGT_DERIV_LINE,
    MODE_TGT_DERIV_VOLUME,
)
from tests._pointsets import sphere_quadrature

GOLDEN = Path(__file__).with_name("golden") / "qbx3d_pairs.json"
PAIR_MODES = {"value": (q.VALUE, 0), "tgt_deriv_1": (None, 1),
              "src_deriv_2": (q.SRC_DERIV_AXIS, 2), "dir_src_deriv": (q.SRC_DERIV_DIR, 0)}


def _golden_cases():
    return json.loads(GOLDEN.read_text())


def test_oracle_matches_sumpy_golden_pairs():
    data = _golden_cases()
    k = data["k"]
    seen = set()
    for c in data["cases"]:
        mode, axis = PAIR_MODES[c["pair"]]
        if mode is None:
            mode = q.TGT_DERIV_LINE if c["expansion"] == "line" else q.TGT_DERIV_VOLUME
        a = np.array(c["avec"])[:, None]
        b = np.array(c["bvec"])[:, None]
        d = np.array(c["dir"])[:, None]
        got = q.pair_values(c["order"], mode, a, b, k if c["kernel"] == "helmholtz" else None,
                            axis, d)[0]
        want = complex(*c["value"])
        assert abs(got - want) <= 2e-14 * abs(want), c
        seen.add((c["kernel"], c["expansion"], c["pair"]))
    # every kernel x expansion x pair combination is pinned
    assert len(seen) == 2 * 3 * 4


def test_oracle_converges_to_kernel():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 20)) + np.array([[0], [0], [3.0]])
    b = 0.3 * rng.standard_normal((3, 20))
    r = np.linalg.norm(a + b, axis=0)
    assert np.abs(q.pair_values(40, q.VALUE, a, b) - 1 / r).max() < 1e-14
    assert np.abs(q.pair_values(60, q.VALUE, a, b, k=2.5) - np.exp(2.5j * r) / r).max() < 1e-14


def test_oracle_derivatives_match_differences():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((3, 8)) + np.array([[0], [0], [2.0]])
    b = 0.4 * rng.standard_normal((3, 8))
    dirs = rng.standard_normal((3, 8))
    h = 1e-6
    for k in (None, 1.7):
        def val(aa, bb):
            return q.pair_values(7, q.VALUE, aa, bb, k)
        e = np.zeros((3, 8))
        e[1] = h
        fd_a = (val(a + e, b) - val(a - e, b)) / (2 * h)
        fd_b = (val(a, b + e) - val(a, b - e)) / (2 * h)
        fd_dir = (val(a + h * dirs, b) - val(a - h * dirs, b)) / (2 * h)
        scale = np.abs(val(a, b)).max()
        assert np.abs(q.pair_values(7, q.TGT_DERIV_LINE, a, b, k, 1) - fd_a).max() < 1e-8 * scale
        assert np.abs(q.pair_values(7, q.TGT_DERIV_VOLUME, a, b, k, 1) - fd_b).max() < 1e-8 * scale
        assert np.abs(q.pair_values(7, q.SRC_DERIV_AXIS, a, b, k, 1) + fd_a).max() < 1e-8 * scale
        assert np.abs(q.pair_values(7, q.SRC_DERIV_DIR, a, b, k, 0, dirs) + fd_dir).max() < \
            1e-8 * scale


def sphere_case(k, ntheta=200, ntargets=4, radius=0.15, order=12):
    """Single layer of cos(theta) and double layer of 1 on the unit sphere,
    QBX centers inside: the interior limits are closed-form (spherical
    Bessel / Hankel functions; k = None is Laplace)."""
    src, w = sphere_quadrature(ntheta)
    tsrc, _ = sphere_quadrature(40)
    tgt = tsrc[:, np.random.default_rng(5).choice(tsrc.shape[1], ntargets, replace=False)]
    ctr = tgt * (1.0 - radius)
    if k is None:
        s_exact = tgt[2] / 3.0
        d_exact = -np.ones(ntargets)
    else:
        j0 = np.sin(k) / k
        j1 = np.sin(k) / k ** 2 - np.cos(k) / k
        h1 = -np.exp(1j * k) * (k + 1j) / k ** 2
        h0p = np.exp(1j * k) * (k + 1j) / k ** 2
        s_exact = 1j * k * h1 * j1 * tgt[2]
        d_exact = 1j * k * k * h0p * j0 * np.ones(ntargets)
    return src, w, tgt, ctr, order, s_exact, d_exact


@pytest.mark.parametrize("k", [None, 2.5])
def test_oracle_sphere_layer_potentials(k):
    src, w, tgt, ctr, order, s_exact, d_exact = sphere_case(k)
    dt = complex if k is not None else float
    s = q.lpot(order, q.VALUE, tgt, ctr, src, (w * src[2]).astype(dt), k, scale=1 / (4 * np.pi))
    d = q.lpot(order, q.SRC_DERIV_DIR, tgt, ctr, src, w.astype(dt), k, dirs=src,
               scale=1 / (4 * np.pi))
    assert np.abs(s - s_exact).max() < 1e-12
    assert np.abs(d - d_exact).max() < 1e-12


def test_layer_potential_host_checks():
    lap, helm = LaplaceKernel(3), HelmholtzKernel(3)
    line = LineTaylorLocalExpansion(lap, 4)
    with pytest.raises(ValueError, match="base kernel"):
        LayerPotential(line, target_kernels=[lap], source_kernels=[helm])
    with pytest.raises(TypeError):
        LayerPotential(line, source_kernels=[lap])
    with pytest.raises(ValueError, match="strength_usage"):
        LayerPotential(line, target_kernels=[lap], source_kernels=[lap], strength_usage=[0, 1])
    lp = LayerPotential(line, target_kernels=[lap, AxisTargetDerivative(0, lap)],
                        source_kernels=[lap, DirectionalSourceDerivative(lap)],
                        strength_usage=[0, 1])
    assert lp.nresults == 2 and lp.strength_count == 2 and lp.name == "qbx_apply"
    assert LayerPotentialMatrixGenerator(line, target_kernels=[lap],
                                         source_kernels=[lap]).name == "qbx_matrix"
    src = np.zeros((3, 4))
    mode = lp._pair_mode(AxisTargetDerivative(2, lap), lap, {}, src)
    assert mode[:2] == (MODE_TGT_DERIV_LINE, 2)
    vol = LayerPotential(VolumeTaylorLocalExpansion(lap, 4), target_kernels=[lap],
                         source_kernels=[lap])
    assert vol._pair_mode(AxisTargetDerivative(1, lap), lap, {}, src)[:2] == \
        (MODE_TGT_DERIV_VOLUME, 1)
    comp = LayerPotential(LinearPDEConformingVolumeTaylorLocalExpansion(lap, 4),
                          target_kernels=[lap], source_kernels=[lap])
    assert not comp.line
    with pytest.raises(NotImplementedError, match="second derivatives"):
        lp._pair_mode(AxisTargetDerivative(0, lap), AxisSourceDerivative(1, lap), {}, src)
    with pytest.raises(TypeError, match="src_derivative_dir"):
        lp._pair_mode(lap, DirectionalSourceDerivative(lap), {}, src)
    with pytest.raises(NotImplementedError):
        LayerPotential(line, target_kernels=[AxisTargetDerivative(0, AxisTargetDerivative(
            1, lap))], source_kernels=[lap])
