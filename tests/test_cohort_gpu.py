"""Subject averaging (CUCorMat's to_average modes) on the GPU against the FP64
oracle: the averaged keys, tau, edge sets and weights are bit-identical."""
import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth

pytestmark = pytest.mark.gpu


def _oracle(bolds, fisher, weighted, mode, value):
    N = bolds[0].shape[1]
    keys = O.cohort_keys(bolds, fisher=fisher, weighted=weighted)
    if mode == "r":
        R, C, V = O.graph_r(keys, N, value, weighted=weighted)
        return keys, R, C, V, value
    R, C, V, tau = O.graph_k(keys, N, O.sparsity_k(N, value), weighted=weighted)
    return keys, R, C, V, tau


def _cohort_graph(ctx, bolds, fisher, weighted, mode, value):
    with ctx.cohort(bolds[0].shape[1], fisher=fisher, weighted=weighted) as c:
        for b in bolds:
            c.add(b)
        g, info = c.graph(mode, value)
        R, C, V = g.to_csr()
        packed = c.packed()
        assert c.subjects == len(bolds)
    return R, C, V, info, packed


@pytest.mark.parametrize("fisher", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("mode,value", [("r", 0.15), ("s", 3.0)])
def test_cohort_exact(ctx, fisher, weighted, mode, value):
    N = 700                                     # not a multiple of the 128-voxel tile
    bolds = [synth.bold_series(N, T, 10, 3000 + T) for T in (150, 97, 33)]   # T not multiples of 16
    keys, Ro, Co, Vo, tau = _oracle(bolds, fisher, weighted, mode, value)
    R, C, V, info, packed = _cohort_graph(ctx, bolds, fisher, weighted, mode, value)
    assert np.array_equal(packed, keys.astype(np.float32))
    assert np.array_equal(R, Ro) and np.array_equal(C, Co)
    if weighted:
        assert np.array_equal(V, Vo)
    else:
        assert V is None
    if mode == "s":
        assert info["tau"] == tau               # the FP64 k-th key, bit for bit
        assert info["edges"] == O.sparsity_k(N, value)


def test_cohort_edge_cases(ctx):
    """Zero-variance voxel, a duplicated voxel (r = 1 up to rounding: the
    r == 1 rule of fisher_trans), an inverted copy (r = -1: -inf, averaged
    key -1), T below one 16-step stage, and ties at tau."""
    N = 300
    bolds = []
    for s, T in enumerate((40, 9, 64)):
        b = synth.bold_series(N, T, 8, 4100 + s)
        b[:, 5] = 3.0                          # constant series
        b[:, 7] = b[:, 6]                      # duplicate
        b[:, 9] = -b[:, 8]                     # inverted copy
        bolds.append(b)
    for fisher in (False, True):
        for weighted in (False, True):
            for mode, value in (("r", 0.2), ("s", 40.0)):
                keys, Ro, Co, Vo, tau = _oracle(bolds, fisher, weighted, mode, value)
                R, C, V, info, packed = _cohort_graph(ctx, bolds, fisher, weighted, mode, value)
                assert np.array_equal(packed, keys.astype(np.float32)), (fisher, weighted, mode)
                assert np.array_equal(R, Ro) and np.array_equal(C, Co), (fisher, weighted, mode)
                if weighted:
                    assert np.array_equal(V, Vo)
                if mode == "s":
                    assert info["tau"] == tau


@pytest.mark.parametrize("s_percent", [7.0, 23.0, 61.0])
def test_cohort_ties_at_tau(ctx, s_percent):
    """Voxels 100..199 repeat voxels 0..99, so every key occurs at least
    twice: the k-th key is tied and the lexicographically first ties are kept
    (FormFullGraph_s's rule)."""
    N = 200
    bolds = []
    for s in range(3):
        b = synth.bold_series(N, 45, 6, 4200 + s)
        b[:, 100:] = b[:, :100]
        bolds.append(b)
    keys, Ro, Co, _, tau = _oracle(bolds, True, False, "s", s_percent)
    assert (keys == tau).sum() >= 2
    R, C, _, info, _ = _cohort_graph(ctx, bolds, True, False, "s", s_percent)
    assert info["tau"] == tau
    assert np.array_equal(R, Ro) and np.array_equal(C, Co)


def test_single_subject_matches_subject_graph(ctx):
    """A cohort of one subject (plain average) is that subject's graph, and so
    is a cohort of two copies ((r + r) / 2 = r)."""
    N, T = 1000, 120
    bold = synth.bold_series(N, T, 10, 555)
    for mode, value in (("r", 0.3), ("s", 2.0)):
        g, info = ctx.build_graph(bold, mode=mode, value=value, sign="signed")
        R0, C0, _ = g.to_csr()
        for copies in (1, 2):
            R, C, _, cinfo, _ = _cohort_graph(ctx, [bold] * copies, False, False, mode, value)
            assert np.array_equal(R, R0) and np.array_equal(C, C0)
            if mode == "s":
                assert cinfo["tau"] == info["tau"]


def test_tiny_cohorts_and_adding_after_graph(ctx):
    for N in (1, 2, 3, 129):
        bolds = [synth.bold_series(N, 20, 2, 60 + N), synth.bold_series(N, 30, 2, 61 + N)]
        keys, Ro, Co, _, _ = _oracle(bolds, True, False, "r", 0.0)
        R, C, _, _, packed = _cohort_graph(ctx, bolds, True, False, "r", 0.0)
        assert np.array_equal(packed, keys.astype(np.float32))
        assert np.array_equal(R, Ro) and np.array_equal(C, Co)
    N = 400
    bolds = [synth.bold_series(N, 50, 6, s) for s in (71, 72, 73)]
    with ctx.cohort(N, fisher=True) as c:
        c.add(bolds[0])
        c.add(bolds[1])
        c.graph("s", 5.0)                     # keys of two subjects
        c.add(bolds[2])                       # keys must be recomputed
        g, info = c.graph("s", 5.0)
        R, C, _ = g.to_csr()
    keys, Ro, Co, _, tau = _oracle(bolds, True, False, "s", 5.0)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co) and info["tau"] == tau


def test_cohort_errors(ctx):
    import pagani
    with ctx.cohort(50) as c:
        with pytest.raises(pagani.PaganiError):
            c.graph("r", 0.3)                 # no subjects yet
        c.add(synth.bold_series(50, 20, 2, 1))
        with pytest.raises(pagani.PaganiError):
            c.graph("s", 150.0)
        with pytest.raises(ValueError):
            c.add(synth.bold_series(49, 20, 2, 1))


def test_large_cohort_of_copies_is_the_subject_graph(ctx):
    """At 20,000 voxels (2 x 10^8 pairs, 1.6 GB accumulator): two copies of a
    subject average to exactly its r, so the cohort's sparsity graph and tau
    equal the subject graph's."""
    N, T = 20000, 150
    bold = synth.bold_series(N, T, 20, 8080)
    g, info = ctx.build_graph(bold, mode="s", value=1.0, sign="signed")
    R0, C0, _ = g.to_csr()
    with ctx.cohort(N) as c:
        c.add(bold)
        c.add(bold)
        gc, cinfo = c.graph("s", 1.0)
        R, C, _ = gc.to_csr()
    assert cinfo["tau"] == info["tau"]
    assert np.array_equal(R, R0) and np.array_equal(C, C0)
