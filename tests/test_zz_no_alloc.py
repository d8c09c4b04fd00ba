"""The allocation-free clustering entry point (pg_clustering_noalloc) for
callers that cannot allocate device memory: its scratch is a static device
array inside the library, so the caller passes only device inputs and
outputs.  Checked against pg_clustering on consecutive calls (the array keeps
the previous call's contents and must be cleared by every call)."""
import numpy as np
import pytest

import pagani
from tests import graphs as G

pytestmark = pytest.mark.gpu


def _call(lib, torch, R, C, stream):
    n = len(R) - 1
    Rd = torch.from_numpy(R).cuda()
    Cd = torch.from_numpy(C).cuda()
    cp = torch.empty(n, dtype=torch.float32, device="cuda")
    tri = torch.empty(n, dtype=torch.int64, device="cuda")
    st = lib.pg_clustering_noalloc(Rd.data_ptr(), Cd.data_ptr(), n, cp.data_ptr(), tri.data_ptr(), stream)
    torch.cuda.synchronize()
    return st, cp.cpu().numpy(), tri.cpu().numpy()


def test_noalloc_matches_pg_clustering_on_consecutive_calls():
    import torch
    lib = pagani.lib()
    stream = torch.cuda.current_stream().cuda_stream
    graphs = [G.from_bold(900, 150, 0.3, 61), G.from_bold(900, 150, 0.3, 61), G.from_bold(700, 120, 0.25, 62)]
    with pagani.Context(0) as ctx:
        for R, C, _ in graphs:
            cp_ref, tri_ref, _ = ctx.clustering(ctx.graph(R, C))
            st, cp, tri = _call(lib, torch, R, C, stream)
            assert st == 0
            assert np.array_equal(tri, tri_ref)      # exact counts, as pg_clustering
            assert np.array_equal(cp, cp_ref)


def test_noalloc_rejects_too_many_nodes():
    import torch
    lib = pagani.lib()
    big = int(lib.pg_clustering_noalloc_max_nodes()) + 1
    R = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.float32, device="cuda")
    assert lib.pg_clustering_noalloc(R.data_ptr(), R.data_ptr(), big, out.data_ptr(), None, None) == 4  # PG_ERR_TOO_LARGE


def _ring_lattice(n, k, extra, seed):
    """n nodes, each joined to its k nearest neighbours on either side (so
    every node is in triangles), plus `extra` random chords; CSR built with
    numpy so that graphs of millions of nodes take seconds."""
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(n, dtype=np.int64), k)
    dst = (src + np.tile(np.arange(1, k + 1), n)) % n
    a = rng.integers(0, n, extra)
    b = rng.integers(0, n, extra)
    src = np.concatenate([src, a])
    dst = np.concatenate([dst, b])
    keep = src != dst
    u = np.concatenate([src[keep], dst[keep]])
    v = np.concatenate([dst[keep], src[keep]])
    key = np.unique(u * n + v)
    rows = key // n
    C = (key % n).astype(np.int32)
    R = np.zeros(n + 1, np.int64)
    np.add.at(R, rows + 1, 1)
    return np.cumsum(R).astype(np.int32), C


def test_noalloc_large_shared_memory_path():
    """n above 393,216 needs more than 48 KB of dynamic shared memory for the
    neighbour bitmap (the opt-in path); two calls in a row."""
    import torch
    lib = pagani.lib()
    stream = torch.cuda.current_stream().cuda_stream
    R, C = _ring_lattice(450_000, 3, 200_000, 63)
    with pagani.Context(0) as ctx:
        cp_ref, tri_ref, _ = ctx.clustering(ctx.graph(R, C))
    for _ in range(2):
        st, cp, tri = _call(lib, torch, R, C, stream)
        assert st == 0
        assert np.array_equal(tri, tri_ref)
        assert np.array_equal(cp, cp_ref)


def test_noalloc_limit_is_reachable():
    """A graph of exactly the advertised number of nodes is accepted (the
    rejection of one node more is the test above)."""
    import torch
    lib = pagani.lib()
    stream = torch.cuda.current_stream().cuda_stream
    nmax = int(lib.pg_clustering_noalloc_max_nodes())
    assert 0 < nmax <= 2_097_150
    R, C = _ring_lattice(nmax, 2, 0, 64)
    st, cp, tri = _call(lib, torch, R, C, stream)
    assert st == 0
    # a ring lattice with two neighbours a side: every node sits in exactly 3
    # triangles among its 4 neighbours, Cp = 3 / 6
    assert np.all(tri == 3)
    assert np.all(cp == np.float32(0.5))
