"""QBX layer potentials on the GPU (sumpy_b200.qbx through the sumpy_qbx_*
C-ABI) against the oracle (oracle/qbx_oracle.py), the unit-sphere closed
forms, and each other (matrix, matrix subset, applier), following sumpy's
test_qbx.py / test_matrixgen.py checks (sumpy/test/test_qbx.py,
sumpy/test/test_matrixgen.py)."""
import numpy as np
import pytest
import torch

from oracle import qbx_oracle as q
from sumpy_b200 import _capi
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
    LayerPotentialMatrixSubsetGenerator,
)
from tests._pointsets import sphere_quadrature
from tests.test_qbx_oracle import sphere_case

pytestmark = pytest.mark.gpu

SCALE = 1.0 / (4.0 * np.pi)
K = 2.5
EXPANSIONS = {"line": LineTaylorLocalExpansion, "volume": VolumeTaylorLocalExpansion,
              "compressed": LinearPDEConformingVolumeTaylorLocalExpansion}


def geometry(ntgt=150, nsrc=400, radius=0.12, seed=0, shell=(0.95, 1.05)):
    """Targets on the unit sphere with centers inside at depth `radius`;
    sources at random directions with radii uniform in `shell`."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((3, nsrc))
    src = g / np.linalg.norm(g, axis=0) * rng.uniform(*shell, nsrc)
    g = rng.standard_normal((3, ntgt))
    tgt = g / np.linalg.norm(g, axis=0)
    ctr = tgt * (1.0 - radius)
    dirs = rng.standard_normal((3, nsrc))
    dirs /= np.linalg.norm(dirs, axis=0)
    return tgt, ctr, src, dirs, np.full(ntgt, radius)


def kernel_pair(name, base):
    return {"value": (base, base, q.VALUE, 0),
            "tgt_deriv": (AxisTargetDerivative(1, base), base, None, 1),
            "src_deriv": (base, AxisSourceDerivative(2, base), q.SRC_DERIV_AXIS, 2),
            "dir_src_deriv": (base, DirectionalSourceDerivative(base), q.SRC_DERIV_DIR, 0)}[name]


def oracle_mode(mode, expansion):
    if mode is None:
        return q.TGT_DERIV_LINE if expansion == "line" else q.TGT_DERIV_VOLUME
    return mode


def rel_err(got, want):
    return np.abs(np.asarray(got) - want).max() / np.abs(want).max()


@pytest.mark.parametrize("helm", [False, True])
@pytest.mark.parametrize("expansion", list(EXPANSIONS))
@pytest.mark.parametrize("pair", ["value", "tgt_deriv", "src_deriv", "dir_src_deriv"])
def test_qbx_matrix_and_lpot_vs_oracle(cuda_device, helm, expansion, pair):
    base = HelmholtzKernel(3) if helm else LaplaceKernel(3)
    order = 9
    tknl, sknl, mode, axis = kernel_pair(pair, base)
    mode = oracle_mode(mode, expansion)
    tgt, ctr, src, dirs, radii = geometry()
    kw = {"src_derivative_dir": dirs} if pair == "dir_src_deriv" else {}
    if helm:
        kw["k"] = K
    k = K if helm else None
    want = q.matrix(order, mode, tgt, ctr, src, k, axis, dirs, SCALE)

    expn = EXPANSIONS[expansion](base, order)
    mat, = LayerPotentialMatrixGenerator(expn, target_kernels=[tknl], source_kernels=[sknl],
                                         device=cuda_device)(None, tgt, src, ctr, radii, **kw)
    assert mat.shape == want.shape
    assert rel_err(mat.cpu().numpy(), want) < 1e-12

    rng = np.random.default_rng(3)
    dens = rng.standard_normal(src.shape[1])
    if helm:
        dens = dens + 1j * rng.standard_normal(src.shape[1])
    res, = LayerPotential(expn, target_kernels=[tknl], source_kernels=[sknl],
                          device=cuda_device)(None, tgt, src, ctr, [dens], radii, **kw)
    assert rel_err(res.cpu().numpy(), want @ dens) < 1e-12

    ti = rng.integers(0, tgt.shape[1], 500)
    si = rng.integers(0, src.shape[1], 500)
    sub, = LayerPotentialMatrixSubsetGenerator(expn, target_kernels=[tknl],
                                               source_kernels=[sknl], device=cuda_device)(
        None, tgt, src, ctr, radii, ti, si, **kw)
    assert rel_err(sub.cpu().numpy(), want[ti, si]) < 1e-12


@pytest.mark.parametrize("helm", [False, True])
def test_qbx_high_order_vs_oracle(cuda_device, helm):
    base = HelmholtzKernel(3) if helm else LaplaceKernel(3)
    tgt, ctr, src, dirs, radii = geometry(ntgt=64, nsrc=256, radius=0.1, seed=4,
                                          shell=(1.0, 1.05))
    k = K if helm else None
    kw = {"k": K} if helm else {}
    for order in (0, 1, 20, 32):
        want = q.matrix(order, q.VALUE, tgt, ctr, src, k, 0, None, SCALE)
        mat, = LayerPotentialMatrixGenerator(
            LineTaylorLocalExpansion(base, order), target_kernels=[base], source_kernels=[base],
            device=cuda_device)(None, tgt, src, ctr, radii, **kw)
        assert rel_err(mat.cpu().numpy(), want) < 1e-11, order


@pytest.mark.parametrize("k", [None, K])
def test_qbx_sphere_layer_potentials(cuda_device, k):
    """Interior limits on the unit sphere, all targets on the GPU: the
    single layer of cos(theta) and the double layer of 1 (closed forms)."""
    src, w, tgt, ctr, order, s_exact, d_exact = sphere_case(k, ntargets=2000)
    base = HelmholtzKernel(3) if k is not None else LaplaceKernel(3)
    kw = {"k": k} if k is not None else {}
    lp = LayerPotential(LineTaylorLocalExpansion(base, order),
                        target_kernels=[base], source_kernels=[
                            base, DirectionalSourceDerivative(base, "normal")],
                        strength_usage=[0, 1], device=cuda_device)
    zero = np.zeros_like(w)
    s, = lp(None, tgt, src, ctr, [w * src[2], zero], None, normal=src, **kw)
    d, = lp(None, tgt, src, ctr, [zero, w], None, normal=src, **kw)
    assert np.abs(s.cpu().numpy() - s_exact).max() < 1e-12
    assert np.abs(d.cpu().numpy() - d_exact).max() < 1e-12


def test_qbx_several_kernels_and_strengths(cuda_device):
    lap = LaplaceKernel(3)
    tgt, ctr, src, dirs, radii = geometry(seed=7)
    rng = np.random.default_rng(8)
    s0, s1 = rng.standard_normal((2, src.shape[1]))
    order = 7
    expn = VolumeTaylorLocalExpansion(lap, order)
    # S s0 + D s1 at the targets, and the z derivative of S s0 + S s1
    lp = LayerPotential(expn, target_kernels=[lap], source_kernels=[
        lap, DirectionalSourceDerivative(lap)], strength_usage=[0, 1], device=cuda_device)
    v, = lp(None, tgt, src, ctr, [s0, s1], radii, src_derivative_dir=dirs)
    want = q.matrix(order, q.VALUE, tgt, ctr, src, scale=SCALE) @ s0 + \
        q.matrix(order, q.SRC_DERIV_DIR, tgt, ctr, src, dirs=dirs, scale=SCALE) @ s1
    assert rel_err(v.cpu().numpy(), want) < 1e-12
    lp2 = LayerPotential(expn, target_kernels=[lap, AxisTargetDerivative(2, lap)],
                         source_kernels=[lap, lap], strength_usage=[0, 0], device=cuda_device)
    v0, v1 = lp2(None, tgt, src, ctr, [s0], radii)
    m0 = q.matrix(order, q.VALUE, tgt, ctr, src, scale=SCALE)
    m1 = q.matrix(order, q.TGT_DERIV_VOLUME, tgt, ctr, src, axis=2, scale=SCALE)
    assert rel_err(v0.cpu().numpy(), 2 * m0 @ s0) < 1e-12
    assert rel_err(v1.cpu().numpy(), 2 * m1 @ s0) < 1e-12


def test_qbx_device_inputs_and_edges(cuda_device):
    lap = LaplaceKernel(3)
    expn = LineTaylorLocalExpansion(lap, 5)
    tgt, ctr, src, dirs, radii = geometry(ntgt=33, nsrc=70, seed=9)
    dev = [torch.as_tensor(x, device=cuda_device) for x in (tgt, ctr, src)]
    lp = LayerPotential(expn, target_kernels=[lap], source_kernels=[lap], device=cuda_device)
    dens = torch.linspace(-1, 1, 70, dtype=torch.float64, device=cuda_device)
    r_dev, = lp(None, dev[0], dev[2], dev[1], [dens], None)
    r_host, = lp(None, tgt, src, ctr, [dens.cpu().numpy()], None)
    assert torch.equal(r_dev, r_host)
    # no targets, no sources
    e, = lp(None, tgt[:, :0], src, ctr[:, :0], [dens], None)
    assert e.shape == (0,)
    z, = lp(None, tgt, src[:, :0], ctr, [dens[:0]], None)
    assert torch.count_nonzero(z) == 0
    sub = LayerPotentialMatrixSubsetGenerator(expn, target_kernels=[lap], source_kernels=[lap],
                                              device=cuda_device)
    empty, = sub(None, tgt, src, ctr, None, np.zeros(0, int), np.zeros(0, int))
    assert empty.shape == (0,)
    with pytest.raises(IndexError):
        sub(None, tgt, src, ctr, None, np.array([0, 33]), np.array([0, 1]))
    with pytest.raises(ValueError, match="order"):
        LineTaylorLocalExpansion(lap, 33)
    out = torch.empty(33, dtype=torch.float64, device=cuda_device)
    t, c, s = dev[0].contiguous(), dev[1].contiguous(), dev[2].contiguous()
    for order, mode, axis in ((33, 0, 0), (4, 7, 0), (4, 1, 3)):
        with pytest.raises(RuntimeError, match="qbx"):
            _capi.call("sumpy_qbx_lpot_laplace_f64", order, mode, axis, 33, _capi.dptr(t), 33,
                       _capi.dptr(c), 33, 70, _capi.dptr(s), 70, None, 70, _capi.dptr(dens),
                       1.0, _capi.dptr(out), _capi.stream_ptr())


def test_qbx_against_sphere_quadrature_convergence(cuda_device):
    """Error of the single layer of cos(theta) falls with the quadrature
    resolution (the QBX coefficients' integrals converge)."""
    lap = LaplaceKernel(3)
    errs = []
    for nt in (60, 100, 160):
        src, w = sphere_quadrature(nt)
        _, _, tgt, ctr, order, s_exact, _ = sphere_case(None, ntheta=12, ntargets=200)
        s, = LayerPotential(LineTaylorLocalExpansion(lap, order), target_kernels=[lap],
                            source_kernels=[lap], device=cuda_device)(
            None, tgt, src, ctr, [w * src[2]], None)
        errs.append(np.abs(s.cpu().numpy() - s_exact).max())
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-8
