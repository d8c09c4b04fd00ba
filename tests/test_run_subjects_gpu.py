"""pg_run_subjects (a cohort through the whole path in one call) against the
individual entry points on the same subjects: identical per-node results and
scalars, surrogates with the documented seeds."""
import numpy as np
import pytest

import pagani
from pagani import synth

pytestmark = pytest.mark.gpu


def test_run_subjects_matches_individual_calls(ctx):
    bolds = [synth.bold_series(400, 80, 6, 501), synth.bold_series(530, 100, 6, 502)]
    res = ctx.run_subjects(bolds, mode="s", value=3.0, sign="abs", n_random=2, swaps_per_edge=2, seed=7)
    lib = pagani.lib()
    for k, (b, r) in enumerate(zip(bolds, res)):
        g, info = ctx.build_graph(b, mode="s", value=3.0, sign="abs")
        assert r["edges"] == info["edges"] and r["tau"] == info["tau"]
        deg, _ = ctx.degree(g)
        assert np.array_equal(r["degree"], deg)
        cp, _, mean = ctx.clustering(g)
        assert np.array_equal(r["cp"], cp) and r["cp_mean"] == mean
        bc, _, eff, lp = ctx.betweenness(g, with_paths=True)
        assert np.array_equal(r["bc"], bc) and np.array_equal(r["eff"], eff) and r["lp"] == lp
        labels, Q, nm = ctx.newman(g)
        assert np.array_equal(r["modules"], labels) and r["Q"] == Q and r["n_modules"] == nm
        m = g.info[1] // 2
        cp_r, lp_r = [], []
        for j in range(2):
            rg, _ = ctx.maslov(g, lib.pg_surrogate_seed(7, k, j), 2 * m)
            cp_r.append(ctx.clustering(rg)[2])
            lp_r.append(ctx.paths(rg)[2])
        gam, lam, sig = pagani.smallworld(mean, cp_r, lp, lp_r)
        assert (r["gamma"], r["lambda"], r["sigma"]) == (gam, lam, sig)


def test_run_subjects_rejects_bad_input(ctx):
    with pytest.raises(pagani.PaganiError):
        ctx.run_subjects([np.zeros((0, 10), np.float32)])


def test_surrogates_replayed_from_a_cuda_graph_match_direct_runs(ctx):
    """The surrogate chain captured once per subject and replayed gives the
    same gamma / lambda / sigma as enqueueing it surrogate by surrogate."""
    bolds = [synth.bold_series(700, 90, 6, 511), synth.bold_series(450, 120, 6, 512)]
    kw = dict(mode="s", value=2.0, sign="abs", n_random=5, swaps_per_edge=10, seed=3, metrics=("cp",))
    a = ctx.run_subjects(bolds, cuda_graphs=True, **kw)
    b = ctx.run_subjects(bolds, cuda_graphs=False, **kw)
    for x, y in zip(a, b):
        assert x["surrogate_graph_replays"] == 4 and y["surrogate_graph_replays"] == 0
        assert (x["gamma"], x["lambda"], x["sigma"]) == (y["gamma"], y["lambda"], y["sigma"])


def test_weighted_run_uses_the_weighted_tools(ctx):
    """build.weighted: strength, Onnela clustering (real and surrogates) and
    the weighted Newman partition, as the individual weighted calls give."""
    bolds = [synth.bold_series(420, 100, 6, 521)]
    res = ctx.run_subjects(bolds, mode="s", value=4.0, sign="abs", n_random=2, swaps_per_edge=2, seed=5,
                           weighted=True, metrics=("degree", "cp", "eff", "modules"))
    r = res[0]
    g, info = ctx.build_graph(bolds[0], mode="s", value=4.0, sign="abs", weighted=True)
    assert r["edges"] == info["edges"]
    deg, _ = ctx.degree(g)
    assert np.array_equal(r["degree"], deg)
    cp, _, mean = ctx.clustering(g, kind="onnela")
    assert np.array_equal(r["cp"], cp) and r["cp_mean"] == mean
    eff, _, lp, _, _ = ctx.paths(g)
    assert np.array_equal(r["eff"], eff) and r["lp"] == lp
    labels, Q, nm = ctx.newman_weighted(g)
    assert np.array_equal(r["modules"], labels) and r["Q"] == Q
    lib = pagani.lib()
    m = g.info[1] // 2
    cp_r, lp_r = [], []
    for j in range(2):
        rg, _ = ctx.maslov(g, lib.pg_surrogate_seed(5, 0, j), 2 * m)
        cp_r.append(ctx.clustering(rg, kind="onnela")[2])
        lp_r.append(ctx.paths(rg)[2])
    assert (r["gamma"], r["lambda"], r["sigma"]) == pagani.smallworld(mean, cp_r, lp, lp_r)
