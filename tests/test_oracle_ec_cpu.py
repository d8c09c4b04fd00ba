"""The eigenvector-centrality oracle (the CUEC tools' power method) pinned
against networkx and a dense symmetric eigensolver: the normalised output is
the leading eigenvector and the reported eigenvalue its eigenvalue."""
import networkx as nx
import numpy as np
import scipy.sparse as sp

from oracle import oracle as O
from tests import graphs as G


def _dense(R, C, V=None):
    n = len(R) - 1
    rows = np.repeat(np.arange(n), np.diff(R))
    vals = np.ones(len(C)) if V is None else V.astype(np.float64)
    return sp.csr_matrix((vals, (rows, C)), shape=(n, n)).toarray()


def test_ec_matches_networkx_direction():
    Gx = nx.gnm_random_graph(80, 400, seed=5)
    A = nx.to_scipy_sparse_array(Gx, nodelist=range(80), format="csr")
    A.sort_indices()
    ec, lam, it, res = O.eigen_centrality(A.indptr.astype(np.int32), A.indices.astype(np.int32))
    ref = nx.eigenvector_centrality_numpy(Gx)
    refv = np.array([ref[i] for i in range(80)])
    assert it < 10000 and res <= 1e-6
    np.testing.assert_allclose(ec / np.linalg.norm(ec), refv / np.linalg.norm(refv), atol=1e-7)
    assert lam == np.float64(lam) and abs(lam - np.linalg.eigvalsh(A.toarray())[-1]) < 1e-6


def test_ec_weighted_eigenpair():
    R, C, V = G.random_weighted(120, 0.08, 2)
    D = _dense(R, C, V)
    w, vecs = np.linalg.eigh(D)
    x, lam, it, res = O.eigen_centrality(R, C, V)
    y, lam2, it2, _ = O.eigen_centrality(R, C, V, raw=True)
    assert it == it2 and lam == lam2
    np.testing.assert_allclose(np.abs(x), np.abs(vecs[:, -1]), atol=1e-7)
    assert abs(lam - w[-1]) < 1e-6 * w[-1]
    # raw output = A x of the same step
    np.testing.assert_allclose(y, D @ x, rtol=1e-12, atol=1e-12)


def test_ec_no_edges_follows_reference_arithmetic():
    R = np.zeros(5, np.int32)
    x, lam, it, res = O.eigen_centrality(R, np.zeros(0, np.int32))
    y, _, _, _ = O.eigen_centrality(R, np.zeros(0, np.int32), raw=True)
    assert it == 2 and lam == 0.0
    assert np.all(np.isnan(x)) and np.all(y == 0.0)
