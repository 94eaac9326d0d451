"""The oracle's interaction-matrix entries (sumpy's P2PMatrixGenerator /
P2PMatrixSubsetGenerator arithmetic) against the oracle's own direct sums,
which are pinned to the reference through the FMM tests: M @ q must equal
the direct sum, with and without exclude_self, Laplace and Helmholtz."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("k", [None, 10.0])
@pytest.mark.parametrize("self_", [False, True])
def test_matrix_times_strengths_is_the_direct_sum(k, self_):
    rng = np.random.default_rng(3)
    src = rng.random((3, 300))
    tgt = src if self_ else rng.random((3, 200))
    tts = np.arange(300) if self_ else None
    m = O.p2p_matrix(tgt, src, tts, helmholtz_k=k)
    assert m.shape == (tgt.shape[1], 300)
    if k is None:
        q = rng.standard_normal(300)
        ref = O.p2p_direct(tgt, src, q, tts)
    else:
        q = rng.standard_normal(300) + 1j * rng.standard_normal(300)
        ref = O.helm_p2p_direct(tgt, src, k, q, tts)
    np.testing.assert_allclose(m @ q, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    if self_:
        assert (np.diag(m) == 0).all()


def test_subset_is_a_selection_of_the_matrix():
    rng = np.random.default_rng(4)
    src, tgt = rng.random((3, 50)), rng.random((3, 40))
    m = O.p2p_matrix(tgt, src, helmholtz_k=3.0)
    it, js = rng.integers(0, 40, 500), rng.integers(0, 50, 500)
    np.testing.assert_array_equal(O.p2p_matrix_entries(tgt, src, it, js, helmholtz_k=3.0),
                                  m[it, js])
