"""Parity at the size the throughput is quoted on: the 58,000-voxel subject
(T = 240, 20 latent signals, seed synthetic.subject_seed(2, 0), |r| ranking)
against the FP64 oracle's results in tests/golden/subject58k.npz
(tests/golden/make_subject58k.py).

Bars: the edge set is the oracle's bit for bit at 0.5 %, 1 % and 2 % for both
Gram precisions (CSR SHA-256, tau and k equal); triangle counts, hop distances
and int64 path counts of 64 fixed sources and Newman labels are identical;
betweenness (FP64 dependencies, summed in another order) within 1e-9
relative, the per-node sum of 1/d and Lp within 1e-12, Q within 1e-9."""
import hashlib
import os

import numpy as np
import pytest

from pagani import synth

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "subject58k.npz")


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def fx():
    return np.load(FIXTURE)


@pytest.fixture(scope="module")
def bold(fx):
    return synth.bold_series(int(fx["N"]), int(fx["T"]), int(fx["signals"]), int(fx["seed"]))


@pytest.fixture(scope="module")
def g1(ctx, bold):
    g, info = ctx.build_graph(bold, mode="s", value=1.0, sign="abs", precision="bf16x3")
    yield g, info
    g.free()


@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_edge_sets_at_three_sparsities(ctx, fx, bold, precision):
    for q, s in enumerate(fx["sparsities"]):
        g, info = ctx.build_graph(bold, mode="s", value=float(s), sign="abs", precision=precision)
        R, C, _ = g.to_csr()
        g.free()
        assert info["edges"] == fx["k"][q]
        assert info["tau"] == fx["tau"][q]
        assert _sha(R, C) == fx["csr_sha256"][q], f"edge set differs at {s}%"
        # the tile error stays far inside the recheck band
        assert info["band_err_max"] < 2e-4


def test_triangles_and_cp(ctx, fx, g1):
    g, _ = g1
    cp, tri, mean = ctx.clustering(g)
    assert _sha(tri) == str(fx["tri_sha256"]) and int(tri.sum()) == int(fx["tri_total"])
    assert mean == pytest.approx(float(fx["cp_mean"]), rel=1e-12)


def test_distances_and_path_counts_of_fixed_sources(ctx, fx, g1):
    g, _ = g1
    dist, sigma = ctx.bfs_sigma(g, fx["sources"])
    for q in range(len(fx["sources"])):
        assert _sha(dist[q]) == fx["dist_sha256"][q]
        assert _sha(sigma[q]) == fx["sigma_sha256"][q]


def test_betweenness_and_path_length(ctx, fx, g1):
    g, _ = g1
    bc, bc64, eff, lp = ctx.betweenness(g, with_paths=True)
    ref = fx["bc"]
    rel = np.max(np.abs(bc64 - ref) / np.maximum(np.abs(ref), 1.0))
    assert rel < 1e-9
    N = int(fx["N"])
    np.testing.assert_allclose(eff, (fx["inv_sum"] / (N - 1)).astype(np.float32), rtol=2e-7)
    assert lp == pytest.approx(float(fx["lp"]), rel=1e-12)


def test_newman_labels_and_q(ctx, fx, g1):
    g, _ = g1
    labels, Q, nm = ctx.newman(g)
    assert nm == int(fx["n_modules"])
    assert np.array_equal(labels, fx["labels"])
    assert Q == pytest.approx(float(fx["Q"]), rel=1e-9)
