"""Small test graphs as CSR (R, C[, V]) numpy arrays, built on the CPU."""
import numpy as np

from oracle import oracle as O
from pagani import synth


def csr_from_edges(n, edges, weights=None):
    adj = [dict() for _ in range(n)]
    for q, (a, b) in enumerate(edges):
        if a == b:
            continue
        w = 1.0 if weights is None else weights[q]
        adj[a][b] = w
        adj[b][a] = w
    R = np.zeros(n + 1, np.int32)
    C, V = [], []
    for i in range(n):
        cols = sorted(adj[i])
        C += cols
        V += [adj[i][c] for c in cols]
        R[i + 1] = R[i] + len(cols)
    C = np.array(C, np.int32)
    V = np.array(V, np.float32)
    return R, C, (V if weights is not None else None)


def from_bold(N, T, thr, seed, signals=10, weighted=False):
    bold = synth.bold_series(N, T, signals, seed)
    z, _ = O.zscore(bold)
    r = O.corr_packed(z, weighted=weighted)
    R, C, V = O.graph_r(r, N, thr, weighted=weighted)
    return R, C, V


def ring_chord(n=8):
    e = [(i, (i + 1) % n) for i in range(n)] + [(0, n // 2)]
    return csr_from_edges(n, e)


def path(n):
    return csr_from_edges(n, [(i, i + 1) for i in range(n - 1)])


def star(n):
    return csr_from_edges(n, [(0, i) for i in range(1, n)])


def two_components_with_isolated():
    e = [(0, 1), (1, 2), (2, 0), (2, 3), (5, 6), (6, 7), (7, 8), (8, 5), (5, 7)]
    return csr_from_edges(10, e)   # nodes 4 and 9 isolated


def complete(n):
    return csr_from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)])


def random_weighted(n, p, seed):
    rng = np.random.default_rng(seed)
    e, w = [], []
    for i in range(n):
        for j in range(i + 1, n):
            if rng.random() < p:
                e.append((i, j))
                w.append(np.float32(rng.uniform(0.2, 1.0)))
    return csr_from_edges(n, e, w)


def bench_like(seed=7):
    """A denser synthetic voxel graph with community structure."""
    return from_bold(1500, 120, 0.3, seed)


def communities(sizes, p_in, p_link, seed):
    """Dense random communities in a chain: G(size, p_in) inside each block,
    G(p_link) between consecutive blocks only, so BFS depth grows with the
    number of blocks while rows stay long."""
    rng = np.random.default_rng(seed)
    n = int(sum(sizes))
    off = np.cumsum([0] + list(sizes))
    edges = []
    for k, sz in enumerate(sizes):
        a = int(off[k])
        m = np.triu(rng.random((sz, sz)) < p_in, 1)
        edges += [(a + int(i), a + int(j)) for i, j in zip(*np.nonzero(m))]
        if k + 1 < len(sizes):
            b = int(off[k + 1])
            m = rng.random((sz, sizes[k + 1])) < p_link
            edges += [(a + int(i), b + int(j)) for i, j in zip(*np.nonzero(m))]
    return csr_from_edges(n, edges)
