#!/usr/bin/env python
"""Writes tests/golden/config1_5000.npz: the reference's OWN CPU pipeline on
the 5,000-voxel single-subject configuration (T = 200, AR(1) + 10 latent
signals, seed synthetic.subject_seed(1, 0), Pearson r > 0.3, binary graph),
compiled from its sources into oracle/_ref/ (oracle/Makefile):

    CorMat_cpu (float z, FP64 dot; the CPU twin of CUCorMat's correlation),
    FormFullGraph r > 0.3 + FormCSRGraph, Cp, APSP_BFS, Betweenness_CPU,
    Partition (Newman, CPU rules).

Run here, where the reference tree is present (under a minute):

    python tests/golden/make_config1.py

Stored: the SHA-256 of the reference CSR, and every pair whose FP64 r (the
oracle's) lies within 1e-6 of 0.3 together with the reference's decision on
it -- the only pairs on which float and FP64 arithmetic may disagree -- then
the reference's per-node Cp floats, mean Cp, nodal efficiency and Lp, float
betweenness and Newman labels.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "pagani-toolkit_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import oracle as O  # noqa: E402
from pagani import synth  # noqa: E402

N, T, SIG, THR = 5000, 200, 10, 0.3


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    O.build(ref=True)
    ref = O.Ref()
    bold = synth.bold_series(N, T, SIG, synth.subject_seed(1, 0))
    cm = ref.cormat_cpu(bold)
    R, C = ref.graph_r(cm, N, np.float32(THR))
    # pairs near the threshold in the FP64 oracle, with the reference's decision
    z, _ = O.zscore(bold)
    r64 = O.corr_packed(z)
    near = np.nonzero(np.abs(r64 - THR) < 1e-6)[0]
    iu = np.triu_indices(N, 1)
    ni, nj = iu[0][near].astype(np.int32), iu[1][near].astype(np.int32)
    ref_keep = (cm[near] > np.float32(THR)).astype(np.int8)
    cp, cp_mean = ref.cp(R, C)
    li, lp = ref.apsp_bfs(R, C)
    bc = ref.betweenness(R, C)
    labels = ref.partition(R, C)
    out = dict(N=N, T=T, signals=SIG, seed=synth.subject_seed(1, 0), thr=THR, edges=len(C) // 2,
               csr_sha256=sha(R, C), near_i=ni, near_j=nj, near_r64=r64[near], near_ref_keep=ref_keep,
               cp=cp, cp_mean=np.float64(cp_mean), li=li, lp=np.float64(lp), bc=bc, labels=labels)
    path = os.path.join(HERE, "config1_5000.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "edges", len(C) // 2, "near pairs", len(near), "modules", labels.max())


if __name__ == "__main__":
    main()
