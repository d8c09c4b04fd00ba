"""The subject-size restatements (oracle/oracle_big.c) give the results of
the pinned small-size restatements in oracle.c: the same edge set, tau and
tie rule as or_graph_k, and or_brandes' betweenness."""
import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth


def _bold_with_ties(N, T, seed):
    b = synth.bold_series(N, T, 8, seed)
    b[:, 5] = b[:, 3]            # identical voxels: r = 1 ties
    b[:, 9] = b[:, 3]
    b[:, 20] = 2.0 * b[:, 11] + 1.0
    b[:, 30] = b[:, 11]
    return b


@pytest.mark.parametrize("abs_mode", [False, True])
def test_topk_equals_graph_k(abs_mode):
    N = 611
    z, _ = O.zscore(_bold_with_ties(N, 97, 4401))
    r = O.corr_packed(z)
    kmax = O.sparsity_k(N, 5.0)
    keys, ii, jj = O.big_topk(z, kmax, abs_mode=abs_mode, threads=3)
    assert len(keys) == kmax
    for s in (0.2, 1.0, 2.0, 5.0):
        k = O.sparsity_k(N, s)
        R, C, _, tau = O.graph_k(r, N, k, abs_mode=abs_mode)
        assert keys[k - 1] == tau
        Rb, Cb = O.csr_from_pairs(N, ii[:k], jj[:k])
        assert np.array_equal(R, Rb) and np.array_equal(C, Cb)


def test_topk_tie_rule_keeps_lexicographically_first():
    # 4 identical voxels and k inside the block of r = 1 ties
    N = 50
    b = synth.bold_series(N, 40, 3, 4402)
    for c in (7, 13, 41):
        b[:, c] = b[:, 2]
    z, _ = O.zscore(b)
    r = O.corr_packed(z)
    for k in (1, 2, 4, 6, 7):
        keys, ii, jj = O.big_topk(z, k, threads=2)
        R, C, _, tau = O.graph_k(r, N, k)
        assert keys[-1] == tau
        Rb, Cb = O.csr_from_pairs(N, ii, jj)
        assert np.array_equal(R, Rb) and np.array_equal(C, Cb)


def test_brandes_mt_equals_brandes():
    from tests import graphs as G
    R, C, _ = G.from_bold(700, 110, 0.3, 4403)
    bc = O.brandes(R, C)
    bc_mt, inv = O.brandes_mt(R, C, threads=5, with_inv_sum=True)
    np.testing.assert_allclose(bc_mt, bc, rtol=1e-12, atol=1e-9)
    inv_o, _, _, _ = O.bfs_paths(R, C)
    assert np.array_equal(inv, inv_o)
