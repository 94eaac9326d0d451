"""GPU interaction-matrix entries (sumpy's P2PMatrixGenerator and
P2PMatrixSubsetGenerator, sumpy/p2p.py:290-477) through the C-ABI against
the oracle's entries: FP64 to 1e-13 relative per entry (the GPU computes
1/r with rsqrt and e^{ikr} with sincos), exclude_self zeros, index subsets,
and M @ q against the GPU direct sum."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sumpy_b200 import (
    P2P,
    HelmholtzKernel,
    LaplaceKernel,
    P2PMatrixGenerator,
    P2PMatrixSubsetGenerator,
)

pytestmark = pytest.mark.gpu


def _kernel(k):
    return LaplaceKernel(3) if k is None else HelmholtzKernel(3)


def _kw(k):
    return {} if k is None else {"k": k}


@pytest.mark.parametrize("k", [None, 10.0])
@pytest.mark.parametrize("self_", [False, True])
@pytest.mark.parametrize("shape", [(1, 1), (37, 300), (515, 129)])
def test_dense_matrix_matches_oracle(cuda_device, k, self_, shape):
    nt, ns = shape
    rng = np.random.default_rng(nt + ns)
    src = rng.random((3, ns))
    tgt = src[:, :nt] if self_ else rng.random((3, nt))
    tts = np.arange(nt) if self_ else None
    (m,) = P2PMatrixGenerator([_kernel(k)], exclude_self=self_)(
        None, tgt, src, target_to_source=tts, **_kw(k))
    ref = O.p2p_matrix(tgt, src, tts, helmholtz_k=k)
    got = m.cpu().numpy()
    assert got.shape == ref.shape
    zero = ref == 0
    np.testing.assert_array_equal(got[zero], 0)
    np.testing.assert_allclose(got[~zero], ref[~zero], rtol=1e-13, atol=0)


@pytest.mark.parametrize("k", [None, 4.0])
def test_subset_matches_oracle_and_dense(cuda_device, k):
    rng = np.random.default_rng(9)
    src, tgt = rng.random((3, 700)), rng.random((3, 650))
    it, js = rng.integers(0, 650, 20000), rng.integers(0, 700, 20000)
    (r,) = P2PMatrixSubsetGenerator([_kernel(k)])(None, tgt, src, tgtindices=it,
                                                  srcindices=js, **_kw(k))
    ref = O.p2p_matrix_entries(tgt, src, it, js, helmholtz_k=k)
    np.testing.assert_allclose(r.cpu().numpy(), ref, rtol=1e-13, atol=0)
    (m,) = P2PMatrixGenerator([_kernel(k)])(None, tgt, src, **_kw(k))
    np.testing.assert_array_equal(r.cpu().numpy(), m.cpu().numpy()[it, js])
    with pytest.raises(IndexError):
        P2PMatrixSubsetGenerator([_kernel(k)])(None, tgt, src, tgtindices=[650],
                                               srcindices=[0], **_kw(k))


def test_matrix_vector_product_is_the_direct_sum(cuda_device):
    rng = np.random.default_rng(2)
    src = rng.random((3, 3000))
    q = rng.standard_normal(3000)
    (m,) = P2PMatrixGenerator([LaplaceKernel(3)], exclude_self=True)(
        None, src, src, target_to_source=np.arange(3000))
    (d,) = P2P([LaplaceKernel(3)], exclude_self=True)(
        None, src, src, (q,), target_to_source=np.arange(3000))
    mq = (m @ torch.as_tensor(q, device="cuda")).cpu().numpy()
    ref = d.cpu().numpy()
    np.testing.assert_allclose(mq, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
