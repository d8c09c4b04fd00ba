"""The oracle restatement against the reference's own CPU functions run live
(oracle/_ref, built from the reference sources where they are present) on
fresh seeded inputs.  CPU only; skipped when the reference build is absent."""
import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth
from tests import graphs as G

pytestmark = pytest.mark.skipif(not O.Ref.available(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def ref():
    return O.Ref()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_graph_and_metrics(ref, seed):
    N, T = 240, 80
    bold = synth.bold_series(N, T, 6, 900 + seed)
    z, _ = O.zscore(bold)
    r = O.corr_packed(z)
    cm = ref.cormat_cpu(bold)
    assert np.max(np.abs(r - cm)) < 1e-6
    R, C, _ = O.graph_r(r, N, 0.25)
    Rr, Cr = ref.graph_r(cm, N, np.float32(0.25))
    near = np.abs(r - 0.25) < 1e-6
    if not near.any():
        assert np.array_equal(R, Rr) and np.array_equal(C, Cr)
    tri, cp, mean = O.cp_binary(R, C)
    cpr, meanr = ref.cp(R, C)
    assert np.array_equal(cp, cpr)
    np.testing.assert_allclose(O.brandes(R, C), ref.betweenness(R, C), rtol=1e-4, atol=1e-3)
    assert np.array_equal(O.newman(R, C)[0], ref.partition(R, C))


@pytest.mark.parametrize("mk", [G.ring_chord, lambda: G.path(40), lambda: G.star(30), G.two_components_with_isolated])
def test_small_graphs(ref, mk):
    R, C, _ = mk()
    np.testing.assert_allclose(O.brandes(R, C), ref.betweenness(R, C), rtol=1e-5, atol=1e-5)
    _, cp, _ = O.cp_binary(R, C)
    assert np.array_equal(cp, ref.cp(R, C)[0])
    inv, _, lp, _ = O.bfs_paths(R, C)
    li, lpr = ref.apsp_bfs(R, C)
    np.testing.assert_allclose(inv / (len(R) - 2), li, rtol=1e-6, atol=1e-7)


def test_ring_chord_betweenness_is_twice_the_undirected_value(ref):
    # an 8-ring with one chord: the reference counts ordered source/target pairs
    R, C, _ = G.ring_chord(8)
    bc = ref.betweenness(R, C)
    assert np.allclose(bc, [15, 5, 2, 5, 15, 5, 2, 5])
    assert np.allclose(O.brandes(R, C), bc)


@pytest.mark.parametrize("seed", [3, 4, 5])
def test_weighted_newman_matches_reference_partition(ref, seed):
    """The weighted tool's CPU Partition (every group split on the CPU rule,
    weights read from the value array by position) against or_newman_weighted
    with the GPU rule never taken."""
    R, C, V = G.from_bold(300, 100, 0.25, 600 + seed, weighted=True)
    res = ref.wpartition(R, C, V)
    if res is None:
        pytest.skip("libref_wnewman.so not built")
    n = len(R) - 1
    lab, Q, nm = O.newman_weighted(R, C, V, gpu_rule_above=n + 1)
    assert np.array_equal(lab, res)
    assert nm == len(np.unique(res))


def test_participation_matches_reference_pc_cpu(tmp_path):
    """The reference's PC_CPU program (oracle/_ref/ref_pc_cpu) on real files.
    It joins paths with a backslash, so the inputs are given names of the form
    'd\\<stem>.csr' in its working directory, beside a directory 'd' that it
    lists."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(O.__file__), "_ref", "ref_pc_cpu")
    if not os.path.exists(exe):
        pytest.skip("ref_pc_cpu not built")
    from tests import graphs as G
    R, C, V = G.from_bold(300, 150, 0.25, 77, weighted=True)
    n = len(R) - 1
    mod = np.random.default_rng(0).integers(1, 9, n).astype(np.float32)
    (tmp_path / "d").mkdir()
    (tmp_path / "d" / "x.csr").write_bytes(b"")
    with open(tmp_path / "d\\x.csr", "wb") as f:
        for a in (np.array([len(R)], np.int32), R, np.array([len(C)], np.int32), C, np.array([len(V)], np.int32), V):
            np.asarray(a).tofile(f)
    with open(tmp_path / "d\\x_modu.nm", "wb") as f:
        np.array([n], np.int32).tofile(f)
        mod.tofile(f)
    subprocess.run([exe, "d"], cwd=tmp_path, capture_output=True, timeout=60)
    pc_ref = np.fromfile(tmp_path / "d\\x_pc.nm", np.int32)[1:].view(np.float32)
    pn_ref = np.fromfile(tmp_path / "d\\x_pc.nm_Normalized.nm", np.int32)[1:].view(np.float32)
    pc, pn, K = O.participation(R, C, V, mod)
    assert np.array_equal(pc, pc_ref) and np.array_equal(pn, pn_ref)


@pytest.mark.parametrize("fisher", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_cohort_average_matches_reference(ref, fisher, weighted):
    """The averaging branch of CUCorMat (post_block with or without
    fisher_trans, division by the subject count, inv_fisher_trans), run by the
    reference's own functions over each subject's float r, against the FP64
    cohort keys of the oracle; the r-threshold graphs agree away from the
    threshold."""
    N = 180
    bolds = [synth.bold_series(N, T, 6, 700 + T) for T in (90, 70, 110)]
    keys = O.cohort_keys(bolds, fisher=fisher, weighted=weighted)
    rs = [O.corr_packed(O.zscore(b)[0], weighted=weighted).astype(np.float32) for b in bolds]
    cm = ref.cohort(rs, N, fisher, weighted)
    tol = 2e-6
    assert np.max(np.abs(cm - keys)) < tol
    thr = 0.2
    R, C, _ = O.graph_r(keys, N, thr)
    Rr, Cr = ref.graph_r(cm, N, np.float32(thr))
    if not (np.abs(keys - thr) < tol).any():
        assert np.array_equal(R, Rr) and np.array_equal(C, Cr)
