"""The C ABI without a GPU: library loads, every declared entry point is
exported, and the host-side logic agrees with the oracle."""
import ctypes as ct
import os
import re

import pytest

import pagani
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pagani.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_[a-z0-9_]+)\s*\(", txt)) - {"pg_log_fn"})


def test_library_exports_every_declared_symbol():
    lib = ct.CDLL(pagani.LIB_PATH)
    missing = [s for s in declared() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_lists_the_header():
    assert sorted(pagani.EXPORTS) == declared()


def test_binding_loads():
    pagani.lib()


@pytest.mark.parametrize("N", [2, 3, 129, 5000, 18500, 46341, 58000, 70000])
@pytest.mark.parametrize("s", [0.001, 0.5, 1.0, 2.0, 5.0, 33.3])
def test_sparsity_edges_matches_oracle(N, s):
    import numpy as np
    assert pagani.sparsity_edges(N, np.float32(s)) == O.sparsity_k(N, np.float32(s))


@pytest.mark.parametrize("M", [0, 1, 15, 16, 17, 1000, 10**6, 16819709])
def test_maslov_round_size_matches_oracle(M):
    assert pagani.maslov_round_size(M) == O.maslov_round_size(M)


def test_smallworld():
    g, l, s = pagani.smallworld(0.5, [0.1, 0.3], 2.0, [1.5, 2.5])
    assert g == pytest.approx(2.5) and l == pytest.approx(1.0) and s == pytest.approx(2.5)


def test_status_strings():
    lib = pagani.lib()
    for st in range(8):
        assert lib.pg_status_string(st)


def test_no_gpu_fails_loudly():
    from tests.conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(pagani.PaganiError):
        pagani.Context(0)


def test_run_opts_defaults_and_surrogate_seeds():
    lib = pagani.lib()
    o = pagani.RunOpts()
    lib.pg_run_opts_default(ct.byref(o))
    b = pagani.BuildOpts()
    lib.pg_build_opts_default(ct.byref(b))
    assert bytes(o.build) == bytes(b)
    assert (o.n_random, o.swaps_per_edge, o.seed) == (0, 2, 1)
    seeds = {lib.pg_surrogate_seed(7, s, r) for s in range(50) for r in range(20)}
    assert len(seeds) == 1000                      # one stream per (subject, surrogate)
    assert lib.pg_surrogate_seed(7, 3, 4) == lib.pg_surrogate_seed(7, 3, 4)
