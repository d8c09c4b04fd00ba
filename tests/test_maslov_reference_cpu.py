"""Maslov-Sneppen surrogates against the reference's own Maslov
(U/cuda_EC/cuda_EC/Maslov.cpp, W/Maslov/Maslov/Maslov.cpp), compiled from its
sources into oracle/_ref/ with rand()/srand() replaced by a seeded 15-bit
generator (oracle/ref_shim/seeded_rand.h).

1. The oracle's sequential Rewire (or_rewire_seq) reproduces the compiled
   reference's surrogates bit for bit, binary and weighted: the swap rule,
   orientation coin, rejection tests and weight re-attachment are pinned.
2. The round schedule the GPU runs (or_maslov, bit-identical to pg_maslov in
   tests/test_metrics_gpu.py) gives the reference's Markov chain: over 100
   seeds at the reference's 2M attempts, the committed fraction and the
   surrogates' mean clustering and path length agree in distribution with
   the reference's own runs (two-sample Kolmogorov-Smirnov, p > 0.01), and
   degrees are preserved."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.skipif(not O.Ref.available(), reason="reference not compiled into oracle/_ref")


def test_sequential_rewire_equals_reference():
    ref = O.Ref()
    R, C, _ = G.from_bold(300, 96, 0.3, 77)
    for seed in (1, 2, 12345):
        Rr, Cr = ref.maslov(R, C, seed)
        Rs, Cs, _, nc = O.rewire_seq(R, C, None, seed)
        assert np.array_equal(Rr, Rs) and np.array_equal(Cr, Cs)
        assert 0 < nc <= len(C)
    Rw, Cw, Vw = G.from_bold(300, 96, 0.25, 78, weighted=True)
    for seed in (3, 4):
        a = ref.maslov(Rw, Cw, seed, V=Vw)
        b = O.rewire_seq(Rw, Cw, Vw, seed)
        assert all(np.array_equal(x, y) for x, y in zip(a, b[:3]))


@pytest.mark.parametrize("N,thr", [(300, 0.3), (500, 0.2)])
def test_round_schedule_matches_reference_distribution(N, thr):
    from scipy import stats
    ref = O.Ref()
    R, C, _ = G.from_bold(N, 96, thr, 77)
    M = len(C) // 2
    deg = np.diff(R)
    a, b = [], []
    for seed in range(1, 101):
        Rr, Cr = ref.maslov(R, C, seed)
        nc = O.rewire_seq(R, C, None, seed)[3]
        Ro, Co, _, no = O.maslov(R, C, None, seed, 2 * M)
        assert np.array_equal(np.diff(Ro), deg)
        a.append((nc / (2 * M), O.cp_binary(Rr, Cr)[2], O.bfs_paths(Rr, Cr)[2]))
        b.append((no / (2 * M), O.cp_binary(Ro, Co)[2], O.bfs_paths(Ro, Co)[2]))
    a, b = np.array(a), np.array(b)
    for k, name in enumerate(("committed fraction", "mean Cp", "Lp")):
        p = stats.ks_2samp(a[:, k], b[:, k]).pvalue
        assert p > 0.01, f"{name}: reference {a[:, k].mean():.5f} vs rounds {b[:, k].mean():.5f} (KS p={p:.4f})"


def test_weighted_values_travel_with_their_edges():
    Rw, Cw, Vw = G.from_bold(300, 96, 0.25, 78, weighted=True)
    Ro, Co, Vo, _ = O.maslov(Rw, Cw, Vw, 9, len(Cw))
    assert np.array_equal(np.sort(Vo), np.sort(Vw))
    rows = np.repeat(np.arange(len(Ro) - 1), np.diff(Ro))
    w = {(int(i), int(j)): float(v) for i, j, v in zip(rows, Co, Vo)}
    assert all(w[(j, i)] == v for (i, j), v in w.items())     # symmetric
