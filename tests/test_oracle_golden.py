"""The oracle restatement against fixtures produced by the reference's own
CPU code (tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_small.npz"))
N = GOLD["bold"].shape[1]


def _pairs(R, C):
    rows = np.repeat(np.arange(len(R) - 1), np.diff(R))
    m = rows < C
    return set(zip(rows[m].tolist(), C[m].tolist()))


def _r_of(r_packed, i, j, n):
    return r_packed[i * n - i * (i + 1) // 2 + (j - i - 1)]


@pytest.fixture(scope="module")
def r64():
    z, nz = O.zscore(GOLD["bold"])
    assert nz == 0
    return O.corr_packed(z)


def test_correlation_matches_reference_cormat(r64):
    # reference: float z-scores, FP64 dot, float store (CorMat.cpp:860-906)
    assert np.max(np.abs(r64 - GOLD["cormat_cpu"])) < 1e-6


def test_r_threshold_graph(r64):
    R, C, _ = O.graph_r(r64, N, 0.3)
    a, b = _pairs(R, C), _pairs(GOLD["r_R"], GOLD["r_C"])
    for (i, j) in a ^ b:   # may differ only where FP64 and the reference's float r straddle 0.3
        assert abs(_r_of(r64, i, j, N) - 0.3) < 1e-6


def test_sparsity_graph_and_tie_rule(r64):
    k = int(GOLD["s_k"])
    assert k == O.sparsity_k(N, 2.0)
    R, C, _, tau = O.graph_k(r64, N, k)
    assert len(C) == 2 * k == len(GOLD["s_C"])
    assert abs(tau - float(GOLD["s_tau"])) < 1e-6
    a, b = _pairs(R, C), _pairs(GOLD["s_R"], GOLD["s_C"])
    for (i, j) in a ^ b:
        assert abs(_r_of(r64, i, j, N) - tau) < 1e-6


def test_abs_threshold_graph(r64):
    R, C, _ = O.graph_r(r64, N, 0.3, abs_mode=True)
    a, b = _pairs(R, C), _pairs(GOLD["abs_R"], GOLD["abs_C"])
    for (i, j) in a ^ b:   # CorMat_CPU accumulates in float
        assert abs(abs(_r_of(r64, i, j, N)) - 0.3) < 1e-5


def test_weighted_graph():
    z, _ = O.zscore(GOLD["bold"])
    r = O.corr_packed(z, weighted=True)
    thr = O.weighted_r_threshold(np.float32(0.25))
    R, C, V = O.graph_r(r, N, thr, weighted=True)
    a, b = _pairs(R, C), _pairs(GOLD["w_R"], GOLD["w_C"])
    for (i, j) in a ^ b:
        assert abs(_r_of(r, i, j, N) - thr) < 1e-6
    if a == b:
        assert np.max(np.abs(V - GOLD["w_V"])) < 1e-6


def test_metrics_on_reference_graph():
    R, C = GOLD["r_R"], GOLD["r_C"]
    bc = O.brandes(R, C)
    np.testing.assert_allclose(bc, GOLD["bc"], rtol=1e-4, atol=1e-3)      # reference: float sigma/delta
    tri, cp, mean = O.cp_binary(R, C)
    assert np.array_equal(cp, GOLD["cp"])                                  # same rounding sequence
    assert mean == pytest.approx(float(GOLD["cp_mean"]), rel=1e-6)
    inv, hist, lp, _ = O.bfs_paths(R, C)
    np.testing.assert_allclose(inv / (N - 1), GOLD["li"], rtol=1e-5, atol=1e-7)   # reference: float sums
    assert lp == pytest.approx(float(GOLD["lp"]), rel=1e-6)
    labels, Q, nm, _ = O.newman(R, C)
    assert np.array_equal(labels, GOLD["labels"])


def test_weighted_metrics_on_reference_graph():
    R, C, V = GOLD["w_R"], GOLD["w_C"], GOLD["w_V"]
    cp, mean = O.onnela(R, C, V, vmax_first_n=True)
    np.testing.assert_allclose(cp, GOLD["onnela"], rtol=1e-5, atol=1e-7)   # reference: float sum
    assert mean == pytest.approx(float(GOLD["onnela_mean"]), rel=1e-5)
    D = np.full((N, N), np.inf, np.float32)
    for i in range(N):
        D[i, C[R[i]:R[i + 1]]] = np.float32(1) / V[R[i]:R[i + 1]]
    np.fill_diagonal(D, 0)
    Do = O.fw_dense(D)
    G = GOLD["fw_dist"]
    fin = np.isfinite(G)
    assert np.array_equal(fin, np.isfinite(Do))
    np.testing.assert_allclose(Do[fin], G[fin], rtol=1e-6)


def test_sparsity_count_formula_matches_reference_float_arithmetic():
    # Clength = (long long)2*M1*s/100.0 with the product in float (CorMat.cpp:310-312)
    assert O.sparsity_k(58000, 1.0) == 16819709
    assert O.sparsity_k(58000, 0.5) == 8409855
    assert O.sparsity_k(5000, 1.0) == 124975


def test_oracle_matches_reference_at_config1_size():
    """The restatement against the reference's own pipeline on the
    5,000-voxel configuration (tests/golden/config1_5000.npz): edge set equal
    except on the listed pairs within 1e-6 of the threshold, and on the
    reference's CSR identical Cp floats and Newman labels, betweenness and
    efficiency within the reference's float accumulation."""
    import os as _os
    fx = np.load(_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "golden", "config1_5000.npz"))
    N = int(fx["N"])
    bold = synth.bold_series(N, int(fx["T"]), int(fx["signals"]), int(fx["seed"]))
    z, _ = O.zscore(bold)
    r = O.corr_packed(z)
    iu = np.triu_indices(N, 1)
    keep = r > float(fx["thr"])
    near = np.zeros(len(r), bool)
    near_idx = fx["near_i"].astype(np.int64) * N - fx["near_i"].astype(np.int64) * (fx["near_i"] + 1) // 2 \
        + fx["near_j"] - fx["near_i"] - 1
    near[near_idx] = True
    assert np.array_equal(r[near_idx], fx["near_r64"])
    keep[near_idx] = fx["near_ref_keep"].astype(bool)          # the reference's decision there
    R, C = O.csr_from_pairs(N, iu[0][keep].astype(np.int32), iu[1][keep].astype(np.int32))
    import hashlib
    h = hashlib.sha256()
    h.update(R.tobytes())
    h.update(C.tobytes())
    assert h.hexdigest() == str(fx["csr_sha256"])
    tri, cp, _ = O.cp_binary(R, C)
    assert np.array_equal(cp, fx["cp"])
    labels, _, _, _ = O.newman(R, C)
    assert np.array_equal(labels, fx["labels"])
    bc, inv = O.brandes_mt(R, C, with_inv_sum=True)
    np.testing.assert_allclose(bc, fx["bc"], rtol=1e-4, atol=1e-2)
    # APSP_BFS sums 1/d over ~5,000 targets in float: up to ~3e-5 relative here
    np.testing.assert_allclose(inv / (N - 1), fx["li"], rtol=1e-4)
