"""The oracle's cohort averaging on the CPU: its FP64 ln and exp against the
C library, the Fisher edge cases, and exact properties of the average."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from pagani import synth


def _ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


def test_ln_within_two_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(1e-17, 1e-10, 500), rng.uniform(0.1, 10, 5000),
                         np.exp(rng.uniform(-700, 700, 2000)), [2.0, 0.5, math.sqrt(2), 1e-300, 5e-324, 1.7e308]])
    got, want = O.fp64_fn("ln", xs), np.log(xs)
    assert _ulps(got, want).max() <= 2.0
    assert O.lib().or_ln(1.0) == 0.0
    assert O.lib().or_ln(0.0) == -math.inf


def test_exp_within_one_ulp():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(-16, 16, 5000), rng.uniform(-700, 700, 2000), [0.0, 1e-20, -1e-20]])
    got, want = O.fp64_fn("exp", xs), np.exp(xs)
    assert _ulps(got, want).max() <= 1.0
    assert O.lib().or_exp(-math.inf) == 0.0


def test_fisher_edges():
    L = O.lib()
    assert L.or_fisher(0.0) == 0.0
    assert L.or_fisher(1.0) == L.or_fisher(1.0 - 1e-6) == pytest.approx(np.arctanh(1 - 1e-6), rel=1e-15)
    assert L.or_fisher(1.0 + 5e-7) == L.or_fisher(1.0)      # weighted range: r in (1, 1+1e-6)
    assert L.or_fisher(-1.0) == -math.inf
    assert L.or_inv_fisher(-math.inf) == -1.0
    r = np.linspace(-0.99, 0.99, 101)
    np.testing.assert_allclose(O.fp64_fn("fisher", r), np.arctanh(r), rtol=1e-14, atol=1e-16)
    z = np.linspace(-8, 8, 101)
    np.testing.assert_allclose(O.fp64_fn("inv_fisher", z), np.tanh(z), rtol=1e-14, atol=1e-15)


def test_one_subject_and_identical_pairs_give_r_exactly():
    N, T = 120, 60
    bold = synth.bold_series(N, T, 5, 31)
    r = O.corr_packed(O.zscore(bold)[0])
    assert np.array_equal(O.cohort_keys([bold]), r)
    assert np.array_equal(O.cohort_keys([bold, bold]), r)          # (r + r) / 2 = r
    assert np.array_equal(O.cohort_keys([bold] * 4), r)            # sums of 4 equal terms are exact


def test_graph_from_cohort_keys_uses_reference_threshold_rules():
    N = 90
    bolds = [synth.bold_series(N, 50, 4, s) for s in (5, 6)]
    keys = O.cohort_keys(bolds, fisher=True)
    k = O.sparsity_k(N, 5.0)
    R, C, _, tau = O.graph_k(keys, N, k)
    assert len(C) == 2 * k and tau == np.sort(keys)[::-1][k - 1]
