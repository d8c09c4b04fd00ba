"""Graph metrics on the GPU against the oracle restatement."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import graphs as G

pytestmark = pytest.mark.gpu

CASES = {
    "ring_chord": G.ring_chord(),
    "path200": G.path(200),
    "star50": G.star(50),
    "islands": G.two_components_with_isolated(),
    "complete30": G.complete(30),
    "bold700": G.from_bold(700, 200, 0.3, 11),
    "bold1500": G.bench_like(),
    # dense enough for the tensor-core Brandes levels (>= 64 neighbours per
    # row): max degree 104 (one 8-bit limb) and 325 (two limbs), depth 6 and 4
    "dense_chain": G.communities([130] * 6, 0.6, 0.03, 1),
    "dense_blocks": G.communities([420, 420, 420], 0.7, 0.004, 2),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request, ctx):
    R, C, _ = CASES[request.param]
    return request.param, R, C, ctx.graph(R, C)


def test_degree(ctx, case):
    name, R, C, g = case
    deg, iso = ctx.degree(g)
    d_or, iso_or = O.degree(R)
    assert np.array_equal(deg, d_or) and iso == iso_or


def test_weighted_strength_bit_exact(ctx):
    R, C, V = G.random_weighted(300, 0.05, 3)
    g = ctx.graph(R, C, V)
    deg, _ = ctx.degree(g)
    d_or, _ = O.degree(R, V)
    assert np.array_equal(deg, d_or)


def test_triangles_and_cp(ctx, case):
    name, R, C, g = case
    cp, tri, mean = ctx.clustering(g)
    tri_or, cp_or, mean_or = O.cp_binary(R, C)
    assert np.array_equal(tri, tri_or)
    assert np.array_equal(cp, cp_or)           # same FP64 rounding sequence
    assert mean == pytest.approx(mean_or, rel=1e-12, abs=1e-15)


def test_paths(ctx, case):
    name, R, C, g = case
    eff, inv, lp, hist, diam = ctx.paths(g, max_hop=256)
    inv_or, hist_or, lp_or, dmax = O.bfs_paths(R, C, max_hop=256)
    assert np.array_equal(hist, hist_or)
    assert diam == dmax
    if dmax <= 64:
        # exact per-distance counts summed as count_d / d, d ascending: the oracle's order
        assert np.array_equal(inv, inv_or)
    else:
        # distances beyond 64 are added as they are found (another order)
        np.testing.assert_allclose(inv, inv_or, rtol=1e-12, atol=0)
    assert lp == pytest.approx(lp_or, rel=1e-12)
    n = len(R) - 1
    np.testing.assert_allclose(eff, (inv_or / max(n - 1, 1)).astype(np.float32), rtol=1e-6)


def test_bfs_sigma_exact(ctx, case):
    name, R, C, g = case
    n = len(R) - 1
    rng = np.random.default_rng(5)
    src = rng.integers(0, n, size=min(n, 40)).astype(np.int32)
    dist, sigma = ctx.bfs_sigma(g, src)
    for q, s in enumerate(src):
        d_or, s_or = O.bfs_source(R, C, int(s))
        assert np.array_equal(dist[q], d_or)
        assert np.array_equal(sigma[q], s_or)


def test_betweenness(ctx, case):
    name, R, C, g = case
    bc, bc64, eff, lp = ctx.betweenness(g, with_paths=True)
    bc_or = O.brandes(R, C)
    np.testing.assert_allclose(bc64, bc_or, rtol=1e-10, atol=1e-9)
    inv_or, _, lp_or, _ = O.bfs_paths(R, C)
    assert lp == pytest.approx(lp_or, rel=1e-12)


def test_newman(ctx, case):
    name, R, C, g = case
    labels, Q, nm = ctx.newman(g)
    lab_or, Q_or, nm_or, _ = O.newman(R, C)
    assert nm == nm_or
    assert np.array_equal(labels, lab_or)
    assert Q == pytest.approx(Q_or, rel=1e-9, abs=1e-12)


def test_fw_unweighted_equals_hops(ctx):
    R, C, _ = G.from_bold(300, 100, 0.35, 4)
    g = ctx.graph(R, C)
    eff, lp, D = ctx.fw_paths(g, want_dist=True)
    n = len(R) - 1
    for s in range(0, n, 37):
        d_or, _ = O.bfs_source(R, C, s)
        ref = np.where(d_or < 0, np.inf, d_or).astype(np.float32)
        assert np.array_equal(D[s], ref)


def test_fw_weighted(ctx):
    R, C, V = G.random_weighted(150, 0.06, 9)
    g = ctx.graph(R, C, V)
    eff, lp, D = ctx.fw_paths(g, want_dist=True)
    n = len(R) - 1
    Dd = np.full((n, n), np.inf, np.float32)
    for i in range(n):
        Dd[i, C[R[i]:R[i + 1]]] = np.float32(1) / V[R[i]:R[i + 1]]
    np.fill_diagonal(Dd, 0)
    D_or = O.fw_dense(Dd)
    fin = np.isfinite(D_or)
    assert np.array_equal(fin, np.isfinite(D))
    np.testing.assert_allclose(D[fin], D_or[fin], rtol=1e-6)
    eff_or, lp_or = O.weighted_paths(R, C, V)
    np.testing.assert_allclose(eff, eff_or, rtol=1e-5)
    assert lp == pytest.approx(lp_or, rel=1e-6)


def test_onnela(ctx):
    R, C, V = G.from_bold(400, 300, 0.2, 21, weighted=True)
    g = ctx.graph(R, C, V)
    for first_n in (False, True):
        cp, _, mean = ctx.clustering(g, kind="onnela", vmax_first_n=first_n)
        cp_or, mean_or = O.onnela(R, C, V, vmax_first_n=first_n)
        np.testing.assert_allclose(cp, cp_or, rtol=1e-5, atol=1e-7)
        assert mean == pytest.approx(mean_or, rel=1e-5)


def test_fw_batched_with_onnela(ctx):
    gs, refs = [], []
    for q, n in enumerate([90, 131, 64, 257]):
        R, C, V = G.from_bold(n, 400, 0.2, 100 + q, weighted=True)
        gs.append(ctx.graph(R, C, V))
        refs.append((R, C, V))
    out = ctx.fw_batched(gs)
    for (eff, lp, cp, cpm), (R, C, V) in zip(out, refs):
        eff_or, lp_or = O.weighted_paths(R, C, V)
        np.testing.assert_allclose(eff, eff_or, rtol=1e-5)
        assert lp == pytest.approx(lp_or, rel=1e-6)
        cp_or, m_or = O.onnela(R, C, V)
        np.testing.assert_allclose(cp, cp_or, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("weighted", [False, True])
def test_maslov_bit_exact(ctx, weighted):
    if weighted:
        R, C, V = G.from_bold(500, 300, 0.2, 31, weighted=True)
    else:
        R, C, V = G.from_bold(600, 200, 0.3, 32)
    g = ctx.graph(R, C, V)
    attempts = 10 * (len(C) // 2)
    g2, committed = ctx.maslov(g, 12345, attempts)
    R2, C2, V2 = g2.to_csr()
    Ro, Co, Vo, comm_or = O.maslov(R, C, V, 12345, attempts)
    assert committed == comm_or
    assert np.array_equal(R2, Ro) and np.array_equal(C2, Co)
    if weighted:
        assert np.array_equal(V2, Vo)
    assert np.array_equal(np.diff(R2), np.diff(R))   # degrees preserved
    n = len(R) - 1
    rows = np.repeat(np.arange(n), np.diff(R2))
    assert not np.any(rows == C2)                    # no self loops
    assert committed > attempts // 20


def _check_ec(ec, lam, it, ec_or, lam_or, it_or):
    """Same step count: values agree to rounding (summation order differs);
    a step count one apart (a borderline stop) still agrees to 1e-4."""
    assert np.array_equal(np.isnan(ec), np.isnan(ec_or))
    ok = ~np.isnan(ec_or)
    if it == it_or:
        np.testing.assert_allclose(ec[ok], ec_or[ok], rtol=1e-9, atol=1e-12 * max(1.0, np.abs(ec_or[ok]).max(initial=0)))
        assert lam == pytest.approx(lam_or, rel=1e-12)
    else:
        assert abs(it - it_or) <= 1
        np.testing.assert_allclose(ec[ok], ec_or[ok], rtol=1e-4, atol=1e-8)


@pytest.mark.parametrize("raw", [False, True])
def test_eigen_centrality(ctx, case, raw):
    name, R, C, g = case
    ec, lam, it, res = ctx.eigen_centrality(g, raw=raw)
    ec_or, lam_or, it_or, res_or = O.eigen_centrality(R, C, raw=raw)
    _check_ec(ec, lam, it, ec_or, lam_or, it_or)


@pytest.mark.parametrize("raw", [False, True])
def test_eigen_centrality_weighted(ctx, raw):
    for R, C, V in (G.random_weighted(300, 0.05, 4), G.from_bold(900, 200, 0.25, 31, weighted=True)):
        g = ctx.graph(R, C, V)
        ec, lam, it, res = ctx.eigen_centrality(g, raw=raw)
        ec_or, lam_or, it_or, res_or = O.eigen_centrality(R, C, V, raw=raw)
        _check_ec(ec, lam, it, ec_or, lam_or, it_or)


def test_eigen_centrality_degenerate(ctx):
    # no edges: the second step normalises a zero vector (0 * inf = NaN in the
    # normalised output, as in the reference); one node; isolated nodes
    for R, C in ((np.zeros(6, np.int32), np.zeros(0, np.int32)),
                 (np.zeros(2, np.int32), np.zeros(0, np.int32)),
                 G.two_components_with_isolated()[:2]):
        g = ctx.graph(R, C)
        for raw in (False, True):
            ec, lam, it, res = ctx.eigen_centrality(g, raw=raw)
            ec_or, lam_or, it_or, res_or = O.eigen_centrality(R, C, raw=raw)
            assert it == it_or
            _check_ec(ec, lam, it, ec_or, lam_or, it_or)


def test_eigen_centrality_subject20k(ctx):
    # a subject graph built on the GPU (20,000 voxels, top 1% |r|)
    from pagani import synth
    bold = synth.bold_series(20000, 240, 20, synth.subject_seed(2, 5))
    g, info = ctx.build_graph(bold, mode="s", value=1.0, sign="abs")
    R, C, _ = g.to_csr()
    ec, lam, it, res = ctx.eigen_centrality(g)
    ec_or, lam_or, it_or, res_or = O.eigen_centrality(R, C)
    _check_ec(ec, lam, it, ec_or, lam_or, it_or)


def test_participation_bit_exact(ctx):
    rng = np.random.default_rng(12)
    cases = [G.from_bold(600, 150, 0.25, 61, weighted=True), G.random_weighted(250, 0.05, 3),
             G.two_components_with_isolated()]
    for R, C, V in cases:
        n = len(R) - 1
        g = ctx.graph(R, C, V)
        for K in (1, 5, 40):
            mod = rng.integers(1, K + 1, n).astype(np.float32)
            pc, pn, k = ctx.participation(g, mod)
            pc_or, pn_or, k_or = O.participation(R, C, V, mod)
            assert k == k_or
            assert np.array_equal(pc, pc_or) and np.array_equal(pn, pn_or)


def test_participation_many_modules_and_newman_labels(ctx):
    # every node its own module (the per-warp sums no longer fit shared
    # memory), and the labels of a Newman partition
    R, C, V = G.from_bold(9000, 60, 0.6, 62, weighted=True)
    n = len(R) - 1
    g = ctx.graph(R, C, V)
    mod = np.arange(1, n + 1, dtype=np.float32)
    pc, pn, k = ctx.participation(g, mod)
    pc_or, pn_or, _ = O.participation(R, C, V, mod)
    assert k == n and np.array_equal(pc, pc_or) and np.array_equal(pn, pn_or)
    Rb, Cb, _ = G.bench_like()
    gb = ctx.graph(Rb, Cb)
    labels, Q, nm = ctx.newman(gb)
    mod = labels.astype(np.float32)
    pc, pn, k = ctx.participation(gb, mod)
    pc_or, pn_or, _ = O.participation(Rb, Cb, None, mod)
    assert k == nm and np.array_equal(pc, pc_or) and np.array_equal(pn, pn_or)


@pytest.mark.parametrize("rule", [25000, 40])
def test_newman_weighted(ctx, rule):
    # rule 25000: every group takes the row rule (the tool's CPU path);
    # rule 40: groups above 40 nodes take the edge rule (its GPU path)
    for R, C, V in (G.from_bold(700, 200, 0.25, 63, weighted=True), G.random_weighted(400, 0.04, 8)):
        g = ctx.graph(R, C, V)
        labels, Q, nm = ctx.newman_weighted(g, gpu_rule_above=rule)
        lab_or, Q_or, nm_or = O.newman_weighted(R, C, V, gpu_rule_above=rule)
        assert nm == nm_or and np.array_equal(labels, lab_or)
        assert Q == pytest.approx(Q_or, abs=1e-12)


def test_newman_weighted_surrogate_uses_original_values(ctx):
    # the tool partitions a random surrogate with the original graph's value array
    R, C, V = G.from_bold(600, 200, 0.25, 64, weighted=True)
    g = ctx.graph(R, C, V)
    s, _ = ctx.maslov(g, 11, len(C))
    Rs, Cs, _ = s.to_csr()
    labels, Q, nm = ctx.newman_weighted(s, weights_of=g)
    lab_or, Q_or, nm_or = O.newman_weighted(Rs, Cs, V)
    assert nm == nm_or and np.array_equal(labels, lab_or)


def test_newman_whole_grid_groups(ctx):
    # a 13,000-voxel graph: the first groups exceed a team's 12,288 rows and
    # run on the whole grid, unweighted and weighted (edge rule above 5,000)
    from pagani import synth
    bold = synth.bold_series(13000, 120, 10, 99)
    g, info = ctx.build_graph(bold, mode="s", value=0.5, sign="abs", weighted=True)
    R, C, V = g.to_csr()
    labels, Q, nm = ctx.newman(g)
    lab_or, Q_or, nm_or, _ = O.newman(R, C)
    assert nm == nm_or and np.array_equal(labels, lab_or)
    labels, Q, nm = ctx.newman_weighted(g, gpu_rule_above=5000)
    lab_or, Q_or, nm_or = O.newman_weighted(R, C, V, gpu_rule_above=5000)
    assert nm == nm_or and np.array_equal(labels, lab_or)


def test_newman_same_result_every_run(ctx):
    """Once every pending group fits a team, groups run as soon as their
    parent is decided, so the order in which they run and end changes from
    call to call.  Labels, Q and every round's log line (iterations,
    residual, eigenvalue) must not: each team's size is a function of its
    group alone and labels are handed out in the reference's round order."""
    from pagani import synth
    bold = synth.bold_series(9000, 120, 10, 1234)
    g, _ = ctx.build_graph(bold, mode="s", value=2.0, sign="abs")
    runs = []
    for _ in range(3):
        log = []
        labels, Q, nm = ctx.newman(g, log=log)
        rounds = [l for l in log if l.startswith("Round:")]
        runs.append((labels, Q, nm, rounds))
    assert any("dependency-driven phase" in l and "(0 groups" not in l for l in log)
    for labels, Q, nm, rounds in runs[1:]:
        assert nm == runs[0][2] and Q == runs[0][1]
        assert np.array_equal(labels, runs[0][0])
        assert rounds == runs[0][3]


def test_dense_brandes_levels_take_the_tensor_core_path(ctx):
    """Per-kernel profiling shows where Brandes ran: a dense graph takes two
    tensor-core launches (levels 2 and 3) and two gather launches per
    128-source batch, a sparse graph only the gather kernel."""
    R, C, _ = CASES["dense_blocks"]
    g = ctx.graph(R, C)
    batches = (len(R) - 1 + 127) // 128
    ctx.profile(True)
    ctx.profile_reset()
    try:
        ctx.betweenness(g)
        nd, msd = ctx.kernel_time("k_bc_dense")
        nb, _ = ctx.kernel_time("k_brandes")
        assert nd == 2 * batches and nb == 2 * batches and msd > 0
        ctx.profile_reset()
        R2, C2, _ = CASES["bold700"]
        ctx.betweenness(ctx.graph(R2, C2))
        assert ctx.kernel_time("k_bc_dense")[0] == 0
        assert ctx.kernel_time("k_brandes")[0] >= 1
    finally:
        ctx.profile(False)


def test_dense_levels_with_split_tail_tiles(ctx):
    """A 20,000-node dense graph has more 128-row tiles (157) than SMs: the
    tiles of the last partial round are split along K and their partial
    path counts summed; sigma and levels stay exact."""
    from pagani import synth
    N = 20000
    bold = synth.bold_series(N, 120, 10, 77)
    g, _ = ctx.build_graph(bold, mode="s", value=2.0, sign="abs")
    R, C, _ = g.to_csr()
    assert R[-1] >= 64 * N                       # dense: the tensor-core levels run
    src = np.random.default_rng(9).integers(0, N, size=40).astype(np.int32)
    ctx.profile(True)
    ctx.profile_reset()
    try:
        dist, sigma = ctx.bfs_sigma(g, src)
        assert ctx.kernel_time("k_bc_dense")[0] == 2
    finally:
        ctx.profile(False)
    for q, s in enumerate(src):
        d_or, s_or = O.bfs_source(R, C, int(s))
        assert np.array_equal(dist[q], d_or)
        assert np.array_equal(sigma[q], s_or)


def test_fw_batched_many_graphs_one_launch(ctx):
    """A batch of 160 weighted ROI graphs of uneven size (from the synthetic
    generator, |r| > 0.2, distances 1/w) in the one-launch FW + Onnela kernel:
    every graph's efficiency, Lp and clustering against the oracle, including
    graphs of one 64-wide block and graphs spanning several k-blocks."""
    rng = np.random.default_rng(404)
    sizes = list(rng.integers(20, 200, size=158)) + [64, 257]
    gs, refs = [], []
    for q, n in enumerate(sizes):
        R, C, V = G.from_bold(int(n), 300, 0.2, 2000 + q, weighted=True)
        gs.append(ctx.graph(R, C, V))
        refs.append((R, C, V))
    out = ctx.fw_batched(gs)
    for (eff, lp, cp, cpm), (R, C, V) in zip(out, refs):
        eff_or, lp_or = O.weighted_paths(R, C, V)
        np.testing.assert_allclose(eff, eff_or, rtol=1e-5)
        assert lp == pytest.approx(lp_or, rel=1e-6)
        cp_or, m_or = O.onnela(R, C, V)
        np.testing.assert_allclose(cp, cp_or, rtol=1e-5, atol=1e-7)
        assert cpm == pytest.approx(m_or, rel=1e-5, abs=1e-9)
