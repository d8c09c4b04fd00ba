"""Network construction on the GPU against the FP64 oracle (bit-exact edge sets)."""
import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth

pytestmark = pytest.mark.gpu


def _oracle_graph(bold, mode, value, sign="signed", weighted=False):
    z, _ = O.zscore(bold)
    r = O.corr_packed(z, weighted=weighted)
    N = bold.shape[1]
    abs_mode = sign == "abs"
    if mode == "r":
        R, C, V = O.graph_r(r, N, value, abs_mode=abs_mode, weighted=weighted)
        return R, C, V, value
    k = O.sparsity_k(N, value)
    R, C, V, tau = O.graph_k(r, N, k, abs_mode=abs_mode, weighted=weighted)
    return R, C, V, tau


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("N,T,mode,value,sign", [
    (700, 200, "r", 0.3, "signed"),
    (1000, 150, "s", 1.0, "signed"),
    (1000, 150, "s", 2.0, "abs"),
    (513, 77, "r", 0.25, "abs"),
    (129, 64, "s", 0.5, "signed"),
])
def test_edge_set_exact(ctx, precision, N, T, mode, value, sign):
    bold = synth.bold_series(N, T, 10, 1000 + N + T)
    g, info = ctx.build_graph(bold, mode=mode, value=value, sign=sign, precision=precision)
    R, C, _ = g.to_csr()
    Ro, Co, _, tau = _oracle_graph(bold, mode, value, sign)
    assert np.array_equal(R, Ro)
    assert np.array_equal(C, Co)
    if mode == "s":
        assert info["tau"] == tau
        assert info["edges"] == O.sparsity_k(N, value)


def test_degree_matches_reference_rule(ctx):
    bold = synth.bold_series(400, 100, 5, 5)
    g, _ = ctx.build_graph(bold, mode="r", value=0.35, precision="fp32")
    R, C, _ = g.to_csr()
    deg, iso = ctx.degree(g)
    d_or, iso_or = O.degree(R)
    assert np.array_equal(deg, d_or) and iso == iso_or


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("mode,value,sign", [("r", 0.3, "signed"), ("s", 1.0, "abs")])
def test_edge_set_exact_with_tight_band(ctx, precision, mode, value, sign):
    # a 1e-4 recheck band still reproduces the FP64 edge set: the tile error of
    # both Gram paths is far below half of it
    N, T = 1200, 240
    bold = synth.bold_series(N, T, 20, 31337)
    g, info = ctx.build_graph(bold, mode=mode, value=value, sign=sign, precision=precision, guard=1e-4)
    R, C, _ = g.to_csr()
    Ro, Co, _, tau = _oracle_graph(bold, mode, value, sign)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_zero_variance_and_duplicate_voxels(ctx, precision):
    # flat series give r = 0 (the reference's NaN -> 0 rule); duplicated
    # series give r at +-1 and go through the range rule in FP64
    bold = synth.bold_series(300, 64, 5, 99)
    bold[:, 5] = 3.0
    bold[:, 17] = bold[:, 3]
    bold[:, 18] = -bold[:, 3]
    for mode, value in (("r", 0.3), ("s", 3.0), ("r", -0.5)):
        g, info = ctx.build_graph(bold, mode=mode, value=value, precision=precision)
        R, C, _ = g.to_csr()
        Ro, Co, _, _ = _oracle_graph(bold, mode, value)
        assert info["zero_variance"] == 1
        assert np.array_equal(R, Ro) and np.array_equal(C, Co)


def test_weighted_values_exact(ctx):
    bold = synth.bold_series(500, 200, 8, 7)
    thr = O.weighted_r_threshold(np.float32(0.2))
    g, _ = ctx.build_graph(bold, mode="r", value=thr, weighted=True, precision="bf16x3")
    R, C, V = g.to_csr()
    z, _ = O.zscore(bold)
    Ro, Co, Vo = O.graph_r(O.corr_packed(z, weighted=True), 500, thr, weighted=True)
    assert np.array_equal(R, Ro) and np.array_equal(C, Co) and np.array_equal(V, Vo)


def test_correlation_packed(ctx):
    bold = synth.bold_series(200, 50, 4, 3)
    r = ctx.correlation_packed(bold)
    z, _ = O.zscore(bold)
    assert np.array_equal(r, O.corr_packed(z).astype(np.float32))


@pytest.mark.parametrize("N", [1, 2, 3, 127, 128, 129, 257])
def test_tiny_and_ragged_sizes(ctx, N):
    bold = synth.bold_series(N, 70, 3, 5 + N)
    for precision in ("fp32", "bf16x3"):
        g, info = ctx.build_graph(bold, mode="s", value=10.0, precision=precision)
        R, C, _ = g.to_csr()
        Ro, Co, _, _ = _oracle_graph(bold, "s", 10.0)
        assert np.array_equal(R, Ro) and np.array_equal(C, Co)


@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_nan_series_give_isolated_voxels(ctx, precision):
    """A voxel with a NaN sample (or NaN everywhere) has a NaN variance: the
    reference's r is NaN there and post_block stores it as 0
    (U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:821), so the voxel has no edge;
    the rest of the graph equals the oracle's."""
    N, T = 500, 120
    bold = synth.bold_series(N, T, 8, 9090)
    bold[:, 17] = np.nan
    bold[40, 123] = np.nan
    bold[:, 300] = np.inf
    z, nz = O.zscore(bold)
    assert nz == 3
    r = O.corr_packed(z)
    for mode, value in (("r", 0.3), ("s", 2.0)):
        g, info = ctx.build_graph(bold, mode=mode, value=value, sign="signed", precision=precision)
        R, C, _ = g.to_csr()
        if mode == "r":
            Ro, Co, _ = O.graph_r(r, N, value)
        else:
            Ro, Co, _, tau = O.graph_k(r, N, O.sparsity_k(N, value))
            assert info["tau"] == tau
        assert info["zero_variance"] == 3
        assert np.array_equal(R, Ro) and np.array_equal(C, Co)
        for v in (17, 123, 300):
            assert R[v + 1] == R[v] or mode == "s"


def test_gram_wait_that_runs_out_returns_timeout_and_context_stays_usable(ctx):
    """Failure path of the tensor-core Gram kernel, with no GPU fault: a test
    hook makes its TMA producer wait 1 ms on an mbarrier that nothing arrives
    on, before any copy or MMA is issued.  Every warp gives up (the waits are
    bounded and abort-aware), TMEM is freed, pg_build_graph returns
    PG_ERR_TIMEOUT, and the same context then builds the graph correctly."""
    import pagani
    N, T = 700, 96
    bold = synth.bold_series(N, T, 6, 4711)
    pagani.lib().pg_debug_stall_next_gram(ctx.h, 1_000_000)
    with pytest.raises(pagani.PaganiError) as e:
        ctx.build_graph(bold, mode="s", value=2.0, sign="signed", precision="bf16x3")
    assert e.value.status == 6                      # PG_ERR_TIMEOUT
    g, info = ctx.build_graph(bold, mode="s", value=2.0, sign="signed", precision="bf16x3")
    R, C, _ = g.to_csr()
    z, _ = O.zscore(bold)
    Ro, Co, _, tau = O.graph_k(O.corr_packed(z), N, O.sparsity_k(N, 2.0))
    assert info["tau"] == tau and np.array_equal(R, Ro) and np.array_equal(C, Co)
