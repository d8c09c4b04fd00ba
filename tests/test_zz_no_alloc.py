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
