"""Generates tests/golden/*.npz from the reference's OWN CPU code.

The reference ships no test vectors for this path (its only "golden" file,
BC_gloden.txt, has no input graph), so the fixtures are produced by running
the reference's CPU functions, compiled from its sources into oracle/_ref/
(oracle/Makefile), on small seeded synthetic inputs.  Run from the repository
root where the reference tree is present:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pagani-toolkit_b200"))

from oracle import oracle as O  # noqa: E402
from pagani import synth  # noqa: E402


def main():
    O.build(ref=True)
    ref = O.Ref()
    out = {}
    # --- correlation and graph construction (U CorMat.cpp, CorMat_CPU.cpp)
    N, T = 300, 96
    bold = synth.bold_series(N, T, 8, 4242)
    out["bold"] = bold
    cm = ref.cormat_cpu(bold)                       # CorMat_cpu: float z, FP64 dot
    out["cormat_cpu"] = cm
    R, C = ref.graph_r(cm, N, np.float32(0.3))      # FormFullGraph + FormCSRGraph, r > 0.3
    out["r_R"], out["r_C"] = R, C
    k = O.sparsity_k(N, 2.0)
    Rs, Cs, tau = ref.graph_s(cm, N, k)             # select + FormFullGraph_s (tie rule)
    out["s_R"], out["s_C"], out["s_tau"], out["s_k"] = Rs, Cs, np.float32(tau), np.int64(k)
    Ra, Ca = ref.graph_abs(ref.cormat_cpu_mt(bold, 2), N, np.float32(0.3))   # CorMat_CPU |r| > 0.3
    out["abs_R"], out["abs_C"] = Ra, Ca
    Rw, Cw, Vw = ref.wgraph_r(cm, N, np.float32(0.25))                      # weighted, r > 0.25 - 1e-6
    out["w_R"], out["w_C"], out["w_V"] = Rw, Cw, Vw
    # --- metrics on the r > 0.3 graph
    bc = ref.betweenness(R, C)
    cp, cpm = ref.cp(R, C)
    li, lp = ref.apsp_bfs(R, C)
    labels = ref.partition(R, C)
    out.update(bc=bc, cp=cp, cp_mean=np.float64(cpm), li=li, lp=np.float64(lp), labels=labels)
    # --- weighted metrics
    cp2, cp2m = ref.cp2(Rw, Cw, Vw)
    d = ref.bfw(Rw, Cw, Vw, 32)
    out.update(onnela=cp2, onnela_mean=np.float64(cp2m), fw_dist=d)
    np.savez_compressed(os.path.join(HERE, "reference_small.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_small.npz"), {k2: np.asarray(v).shape for k2, v in out.items()})


if __name__ == "__main__":
    main()
