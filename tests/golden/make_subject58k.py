#!/usr/bin/env python
"""Writes tests/golden/subject58k.npz: the FP64 oracle's results on the
58,000-voxel subject that bench.py measures (N = 58,000, T = 240, 20 latent
signals, seed synthetic.subject_seed(2, 0), |r| ranking), so that the GPU path
can be checked at the size its throughput is quoted on.

Run here, on the CPU (about an hour on 8 cores: the pair selection is two
vectorised passes over the 1.68e9 pairs, betweenness is all-source Brandes on
8 threads, Newman runs single-threaded):

    python tests/golden/make_subject58k.py [--voxels N] [--out PATH]

The fixture holds, for sparsities 0.5 %, 1 % and 2 % (k from the reference's
float formula): k, tau and the SHA-256 of the CSR row offsets and columns
(int32 little-endian); at 1 %: the SHA-256 of the exact triangle counts, the
mean Cp, the Newman labels, Q and module count, FP64 betweenness of every
node, the per-node sum of 1/d (efficiency and Lp), and for 64 fixed sources
the SHA-256 of their hop distances and exact int64 path counts.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "pagani-toolkit_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import oracle as O  # noqa: E402
from pagani import synth  # noqa: E402

SPARSITIES = (0.5, 1.0, 2.0)
T_LEN, N_SIG = 240, 20


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def fixed_sources(N, count=64):
    rng = np.random.Generator(np.random.PCG64(58064))
    return np.sort(rng.choice(N, size=count, replace=False)).astype(np.int32)


def log(msg, t0):
    print(f"[{time.time() - t0:8.1f} s] {msg}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--voxels", type=int, default=58000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    N = a.voxels
    out = a.out or os.path.join(HERE, "subject58k.npz" if N == 58000 else f"subject{N}.npz")
    t0 = time.time()
    bold = synth.bold_series(N, T_LEN, N_SIG, synth.subject_seed(2, 0))
    z, zero = O.zscore(bold)
    ks = [O.sparsity_k(N, s) for s in SPARSITIES]
    keys, ii, jj = O.big_topk(z, max(ks), abs_mode=True, threads=a.threads)
    log(f"selection of {len(keys)} pairs", t0)
    fx = {"N": N, "T": T_LEN, "signals": N_SIG, "seed": synth.subject_seed(2, 0), "zero_variance": zero,
          "sparsities": np.array(SPARSITIES), "k": np.array(ks, np.int64),
          "tau": np.array([keys[k - 1] for k in ks]),
          "csr_sha256": np.array([sha(*O.csr_from_pairs(N, ii[:k], jj[:k])) for k in ks])}
    k1 = ks[SPARSITIES.index(1.0)]
    R, C = O.csr_from_pairs(N, ii[:k1], jj[:k1])
    del keys, ii, jj
    tri, cp, cp_mean = O.cp_binary(R, C)
    fx.update(tri_sha256=sha(tri), tri_total=int(tri.sum()), cp_mean=cp_mean)
    log("triangles", t0)
    src = fixed_sources(N)
    d_sha, s_sha = [], []
    for s in src:
        dist, sigma = O.bfs_source(R, C, int(s))
        assert sigma.min() >= 0
        d_sha.append(sha(dist))
        s_sha.append(sha(sigma))
    fx.update(sources=src, dist_sha256=np.array(d_sha), sigma_sha256=np.array(s_sha))
    log("64 single-source BFS", t0)
    # Newman on one thread while betweenness uses the rest
    import threading
    res = {}

    def newman():
        res["newman"] = O.newman(R, C)
        log("newman", t0)

    th = threading.Thread(target=newman)
    th.start()
    bc, inv = O.brandes_mt(R, C, threads=max(1, a.threads - 1), with_inv_sum=True)
    log("betweenness", t0)
    th.join()
    labels, Q, nm, _ = res["newman"]
    total = float(inv.sum())
    fx.update(bc=bc, inv_sum=inv, lp=N * (N - 1) / total if total > 0 else 0.0, labels=labels, Q=Q, n_modules=nm)
    np.savez_compressed(out, **fx)
    log(f"wrote {out}", t0)


if __name__ == "__main__":
    main()
