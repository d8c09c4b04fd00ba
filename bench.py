#!/usr/bin/env python
"""Throughput of the PAGANI hot path on B200: one step = one full subject.

Workload (the 58k-voxel single-subject configuration): N = 58,000 masked
voxels, T = 240 float32 samples, AR(1) phi = 0.5 + 20 latent signals
(seeded synthetic series -- no dataset is distributed with the reference),
top 1% of |r| off-diagonal pairs kept (sparsity mode), then degree,
clustering coefficient (exact triangles), hop path length + nodal
efficiency, Brandes betweenness from all sources (fused with the path
sweep) and Newman leading-eigenvector modularity.

  value  -- subjects/min with the series already resident in HBM (device
            input pointer), all ranks together;
  e2e    -- the same through the C ABI with the series in pinned host memory:
            the host->device copy of the series and the device->host copy of
            every per-node result are inside the timed region.
  roofline -- the dominant kernel, k_brandes (Brandes gather sweeps), timed
            with CUDA events around its launches during the timed steps
            (pg_profile_*), against the algorithmic bytes of its backward sweep
            and the measured HBM copy peak; tensor_levels gives the same for
            k_bc_dense (Brandes levels 2-3 as int8 tensor-core GEMMs, one pass
            over the dense adjacency per launch).
  extras -- eigenvector centrality and subject averaging (FP64 cohort Gram
            with the Fisher transform) on the same subject, outside the step.

--impl reference times the reference's own CPU code of the path (compiled
from its sources into oracle/_ref/) on the host cores; see cpu_baseline().

Multi-GPU: subjects are independent, so N GPUs run N replicas (one subject
stream each, no collective on the data path); the step time is the maximum
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pagani-toolkit_b200"))

import numpy as np  # noqa: E402

N_VOX, T_LEN, N_SIG, SPARSITY = 58000, 240, 20, 1.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, one-pass ncu
# capture) of the k_brandes launches of one 128-source batch (the level-1
# launch and the resumed launch) on the 58000-voxel subject; the workload is
# deterministic, so it holds for every run
BRANDES_DRAM_BYTES_PER_BATCH_58K = 1.127e9
WORKLOAD = "subject-58k: N=58000 voxels, T=240, 20 latent signals, top 1% |r| -> binary CSR; " \
           "degree, Cp (triangles), Lp/efficiency, Brandes BC all sources, Newman modularity"


# --------------------------------------------------------------- helpers
def set_voxels(n):
    global N_VOX, WORKLOAD
    if n != N_VOX:
        WORKLOAD = WORKLOAD.replace(f"N={N_VOX}", f"N={n}").replace("subject-58k", f"subject-{n}")
        N_VOX = n


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def reduce_max_ms(t_ms, device):
    """Step time of a multi-rank run: the maximum over ranks (replicas)."""
    import torch
    import torch.distributed as dist
    tt = torch.tensor([t_ms], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spawned(local, world, port, fn, fn_args):
    os.environ.update(RANK=str(local), LOCAL_RANK=str(local), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    fn(*fn_args)


def spawn_ranks(world, fn, *fn_args):
    """Start `world` ranks of fn(*fn_args) on this node, one process each, with
    RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT set as torchrun
    sets them (used when bench.py --gpus N is started without torchrun)."""
    import torch.multiprocessing as mp
    mp.spawn(_spawned, args=(world, _free_port(), fn, fn_args), nprocs=world, join=True)


def rank_subject_seed(rank):
    """Every replica processes its own subject stream."""
    from pagani import synth
    return synth.subject_seed(2, rank)


# ----------------------------------------------------- reference CPU arm
class _Quiet:
    """Silences the reference's console output (it prints per round/source)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def cpu_baseline(n_sample=4000, threads=None):
    with _Quiet():
        return _cpu_baseline(n_sample, threads)


def _cpu_stage_times(ref, O, synth, n, threads):
    """Seconds per stage of the reference's CPU pipeline on a complete
    n-voxel subject (same generator, T and density as the benchmark)."""
    bold = synth.bold_series(n, T_LEN, N_SIG, synth.subject_seed(2, 99))
    st = {}
    t = time.perf_counter()
    cm = ref.cormat_cpu_mt(bold, threads)
    st["correlation"] = time.perf_counter() - t
    k = O.sparsity_k(n, SPARSITY)
    t = time.perf_counter()
    R, C, _ = ref.graph_s(np.abs(cm), n, k)
    st["threshold_csr"] = time.perf_counter() - t
    t = time.perf_counter()
    ref.cp(R, C)
    st["cp"] = time.perf_counter() - t
    t = time.perf_counter()
    ref.apsp_bfs(R, C)
    st["paths"] = time.perf_counter() - t
    t = time.perf_counter()
    ref.betweenness(R, C)
    st["betweenness"] = time.perf_counter() - t
    t = time.perf_counter()
    ref.partition(R, C)
    st["newman"] = time.perf_counter() - t
    return st


def _cpu_baseline(n_sample=4000, threads=None):
    """The reference's own CPU pipeline (oracle/_ref) on a down-scaled subject.

    The reference CPU code cannot run the 58k subject in bounded time
    (single-thread Brandes alone is hours; CorMat_cpu_MT overflows its int
    pair index beyond ~18.5k voxels).  The sample is a complete subject with
    the same generator, T and density at n_sample voxels; each stage's time
    is scaled to N = 58,000 by its work: N^2 for the correlation, selection
    and CSR build, N^3 (fixed density, so N * nnz) for clustering, BFS path
    length, betweenness and modularity.  A second complete subject of half
    the size checks those exponents: the measured exponent of every stage
    (log of the time ratio over log 2) is reported beside the assumed one.
    """
    from oracle import oracle as O
    from pagani import synth
    threads = threads or os.cpu_count() or 1
    os.environ["PAGANI_REF_THREADS"] = str(threads)
    ref = O.Ref()
    half = _cpu_stage_times(ref, O, synth, n_sample // 2, threads)
    st = _cpu_stage_times(ref, O, synth, n_sample, threads)
    quad = ("correlation", "threshold_csr")
    exps = {k2: (2 if k2 in quad else 3) for k2 in st}
    measured = {k2: (float(np.log(st[k2] / half[k2]) / np.log(2.0)) if half[k2] > 0 and st[k2] > 0 else None)
                for k2 in st}
    sec = sum(st[k2] * (N_VOX / n_sample) ** exps[k2] for k2 in st)
    return {
        "value": 60.0 / sec, "unit": "subjects/min", "cores": threads, "kind": "reference",
        "sample": f"reference CPU pipeline (CorMat_cpu_MT, FormFullGraph_s on |r|, FormCSRGraph, Cp, APSP_BFS, "
                  f"Betweenness_CPU, Partition) on a complete N={n_sample} subject, T={T_LEN}, top 1%; stage "
                  f"times scaled to N={N_VOX} by N^2 (correlation/threshold) and N^3 (graph metrics); "
                  f"measured sample seconds " + json.dumps({k2: round(v, 3) for k2, v in st.items()}),
        "extrapolated_seconds_per_subject": sec,
        "exponent_check": {"half_sample_voxels": n_sample // 2,
                           "half_sample_seconds": {k2: round(v, 3) for k2, v in half.items()},
                           "assumed": exps,
                           "measured": {k2: (round(v, 2) if v is not None else None) for k2, v in measured.items()},
                           "extrapolated_seconds_with_measured_exponents": float(sum(
                               st[k2] * (N_VOX / n_sample) ** (measured[k2] if measured[k2] is not None else exps[k2])
                               for k2 in st))},
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_baseline()
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline())
    wall = time.perf_counter() - t0
    v = float(np.median([x["value"] for x in vals]))
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": "cohort subjects/min @58k voxels", "value": v, "unit": "subjects/min", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1000 / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic", "impl": "reference", "config": {"workload": WORKLOAD},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "subjects/min", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



# ------------------------------------------------- precision report (config 3)
FIXTURE_58K = os.path.join(ROOT, "tests", "golden", "subject58k.npz")
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # FP32 lanes x FMA x max clock


def _sha(*arrays):
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def precision_report(ctx, bold_dev, last):
    """The 58k subject against the FP64 oracle's results committed in
    tests/golden/subject58k.npz: edge sets at 0.5 / 1 / 2 % for both Gram
    precisions (SHA-256 of the CSR, tau, k), the tile error |r_tile - r| over
    the FP64 recheck band, and the relative errors of the timed step's
    betweenness, Q and Lp."""
    if N_VOX != 58000 or not os.path.exists(FIXTURE_58K):
        return None
    fx = np.load(FIXTURE_58K)
    rep = {"oracle": "FP64 restatement (tests/golden/subject58k.npz)", "edge_sets": {}}
    for prec in ("bf16x3", "fp32"):
        rows = []
        for q, s in enumerate(fx["sparsities"]):
            g, info = ctx.build_graph(None, mode="s", value=float(s), sign="abs", precision=prec,
                                      device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
            R, C, _ = g.to_csr()
            g.free()
            rows.append({"sparsity_percent": float(s), "k": int(fx["k"][q]), "edges": info["edges"],
                         "tau_equal": info["tau"] == float(fx["tau"][q]),
                         "edge_set_identical": _sha(R, C) == str(fx["csr_sha256"][q]),
                         "band_pairs": info["band_pairs"], "band_err_max": info["band_err_max"],
                         "band_err_mean": info["band_err_mean"]})
        rep["edge_sets"][prec] = rows
    bc_ref = fx["bc"]
    rep["bc_rel_err_max"] = float(np.max(np.abs(last["bc64"] - bc_ref) / np.maximum(np.abs(bc_ref), 1.0)))
    rep["Q_rel_err"] = abs(last["Q"] - float(fx["Q"])) / abs(float(fx["Q"]))
    rep["newman_labels_identical"] = bool(np.array_equal(last["labels"], fx["labels"]))
    rep["lp_rel_err"] = abs(last["lp"] - float(fx["lp"])) / float(fx["lp"])
    rep["timed_step_edges_and_tau_equal"] = (last["nnz"] // 2 == int(fx["k"][1]) and
                                             last["build"]["tau"] == float(fx["tau"][1]))
    return rep


def build_stage(ctx, bold_dev, stream, hbm_peak, bf16_peak, reps=5):
    """Network construction alone for each Gram precision (CUDA events around
    pg_build_graph with the series on the device, after one warm-up), and the
    emit pass's arithmetic rate: 2*M1*T useful flop per product (3 products
    in split-BF16) against the measured bf16 tensor peak, or against the
    nominal FP32 SIMT peak for the FP32 path."""
    import torch
    M1 = N_VOX * (N_VOX - 1) // 2
    out = {}
    for prec in ("bf16x3", "fp32"):
        kw = dict(mode="s", value=SPARSITY, sign="abs", precision=prec, device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
        g, info = ctx.build_graph(None, **kw)
        g.free()
        ms, emit, hist = [], [], []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g, info = ctx.build_graph(None, **kw)
            e1.record(stream)
            torch.cuda.synchronize()
            g.free()
            ms.append(e0.elapsed_time(e1))
            emit.append(info["ms_emit"])
            hist.append(info["ms_hist"])
        emit_ms = float(np.median(emit))
        products = 3 if prec == "bf16x3" else 1
        tflops = products * 2.0 * M1 * T_LEN / (emit_ms / 1000.0) / 1e12
        peak = bf16_peak if prec == "bf16x3" else FP32_SIMT_NOMINAL_TFLOPS
        out[prec] = {"ms_build": float(np.median(ms)), "ms_gram_hist_passes": float(np.median(hist)),
                     "ms_gram_emit_pass": emit_ms, "kernel": "k_gram_tc" if prec == "bf16x3" else "k_gram_simt",
                     "emit_tflops": tflops, "peak_tflops": peak,
                     "peak_source": "measured bf16 (MEASURED_PEAKS.json)" if prec == "bf16x3"
                     else "nominal FP32 SIMT (148 SMs x 128 lanes x 2 x 1.965 GHz)",
                     "frac": tflops / peak}
    out["split_bf16_speedup_vs_fp32"] = out["fp32"]["ms_build"] / out["bf16x3"]["ms_build"]
    return out


# ----------------------------------------------------------- cohort (config 5)
COHORT_N, COHORT_T, COHORT_SPARSITY, COHORT_RANDOM, COHORT_SWAPS = (40000, 70000), (150, 240), 0.5, 20, 10


def cohort_subjects(count, rank=0):
    """Subjects of the 64-subject cohort configuration, drawn in order from one
    seeded stream: N ~ U{40k..70k}, T ~ U{150..240}, 20 latent signals."""
    from pagani import synth
    rng = np.random.Generator(np.random.PCG64(synth.subject_seed(5, 500 + rank)))
    out = []
    for k in range(count):
        n = int(rng.integers(COHORT_N[0], COHORT_N[1] + 1))
        t = int(rng.integers(COHORT_T[0], COHORT_T[1] + 1))
        out.append((n, t, synth.subject_seed(5, 64 * rank + k)))
    return out


def cohort_leg(ctx, count, rank=0):
    """pg_run_subjects on `count` subjects of the cohort configuration, series
    in pinned host memory (the copy to the device is inside the time): build
    at 0.5 %, degree, Cp, hop Lp / efficiency, 20 Maslov surrogates with
    10 x |E| attempts each (clustering and Lp of every surrogate, CUDA-graph
    replays) and sigma.  Wall time per subject around the call (it returns
    after its results are on the host)."""
    import torch
    from pagani import synth
    subs = cohort_subjects(count, rank)
    series = [torch.from_numpy(synth.bold_series(n, t, N_SIG, sd)).pin_memory() for n, t, sd in subs]
    res = {}
    for prec in ("bf16x3", "fp32"):
        kw = dict(mode="s", value=COHORT_SPARSITY, sign="abs", n_random=COHORT_RANDOM, swaps_per_edge=COHORT_SWAPS,
                  seed=5, metrics=("degree", "cp", "eff"), precision=prec)
        # warm-up: one surrogate per subject, so that every shape bucket is
        # tuned (autotuner cache) and the workspace sized before timing
        warm = dict(kw, n_random=1)
        for b in series:
            ctx.run_subjects([b.numpy()], **warm)
        secs, sig = [], []
        for b in series:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = ctx.run_subjects([b.numpy()], **kw)[0]
            secs.append(time.perf_counter() - t0)
            sig.append({"sigma": r["sigma"], "gamma": r["gamma"], "lambda": r["lambda"], "edges": r["edges"],
                        "replays": r["surrogate_graph_replays"]})
        res[prec] = {"subjects_per_min": 60.0 * len(secs) / sum(secs), "s_per_subject": secs, "results": sig}
    res["subjects"] = [{"N": n, "T": t} for n, t, _ in subs]
    res["workload"] = (f"cohort sample: {count} of the 64 subjects (N ~ U{{40k..70k}}, T ~ U{{150..240}}), top 0.5% "
                       f"|r|, degree, Cp, Lp/efficiency, {COHORT_RANDOM} Maslov surrogates x {COHORT_SWAPS}|E| "
                       "attempts with Cp and Lp each, gamma/lambda/sigma; series from pinned host memory")
    return res


# ------------------------------------------------- weighted ROI batch (config 4)
ROI_GRAPHS, ROI_N, ROI_T, ROI_R = 512, (90, 1024), 1200, 0.2


def roi_batch_leg(ctx, stream, reps=3):
    """512 ROI-level graphs, n ~ U{90..1024}, T = 1200, weight r for r > 0.2
    (the weighted tool's rule), distance 1/w: blocked Floyd-Warshall APSP
    (FP32 min-plus) and Onnela clustering of all graphs in one cooperative
    launch (pg_fw_batched), CUDA events around the call after a warm-up
    (graphs built beforehand).  FP32 roofline: 2 operations (add, min) per
    (i, j, k) update, useful updates sum n^3, against the nominal FP32 rate."""
    import torch
    from pagani import synth
    series = synth.roi_batch(ROI_GRAPHS, ROI_N[0], ROI_N[1], ROI_T, N_SIG, synth.subject_seed(4))
    t0 = time.perf_counter()
    graphs = [ctx.build_graph(b, mode="r", value=ROI_R, sign="signed", weighted=True)[0] for b in series]
    build_s = time.perf_counter() - t0
    ctx.fw_batched(graphs)                       # warm-up (autotuner, workspace)
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = ctx.fw_batched(graphs)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    ctx.profile(True)
    ctx.profile_reset()
    ctx.fw_batched(graphs)
    k_launches, k_ms = ctx.kernel_time("k_fw_batch")
    ctx.profile(False)
    sizes = np.array([b.shape[1] for b in series], np.float64)
    padded = np.ceil(sizes / 64.0) * 64.0
    updates = float(np.sum(sizes ** 3))
    t = float(np.median(ms))
    for g in graphs:
        g.free()
    return {"graphs": ROI_GRAPHS, "n_range": list(ROI_N), "T": ROI_T, "ms_fw_onnela_call": t,
            "ms_kernel": k_ms / max(1, k_launches), "kernel": "k_fw_batch",
            "graphs_per_s": ROI_GRAPHS / (t / 1000.0), "useful_updates": updates,
            "padded_updates": float(np.sum(padded ** 3)),
            "fp32_ops_per_s_tera": 2.0 * updates / (k_ms / max(1, k_launches) / 1000.0) / 1e12,
            "frac_of_nominal_fp32": 2.0 * updates / (k_ms / max(1, k_launches) / 1000.0) / 1e12
            / FP32_SIMT_NOMINAL_TFLOPS,
            "s_graph_builds": build_s, "lp_mean": float(np.mean([o[1] for o in out])),
            "cp_mean": float(np.mean([o[3] for o in out]))}


# ------------------------------------------------------- profiling cases
def kernel_case(args):
    """One small workload of one kernel family, for ncu captures (the metric
    is not quoted on these): builds the subject of --voxels voxels (T = 240,
    20 signals) and runs the case's call once after a warm-up call.
      paths    -- hop paths of a Maslov surrogate at 0.5 % (k_msbfs_all)
      maslov   -- one rewiring of 10 x |E| attempts at 0.5 % (k_ms_rounds)
      fw_batch -- FW + Onnela of --graphs ROI graphs, n ~ U{90..1024} (k_fw_batch)
      gram     -- one split-BF16 build at 1 % (k_gram_tc)
      brandes  -- betweenness at 1 % (k_brandes, k_bc_dense)
      newman   -- modularity at 1 % (k_nm_grid, k_nm_team)
    Prints one JSON line with the call's device time."""
    import torch
    import pagani
    from pagani import synth
    ctx = pagani.Context(0)
    stream = torch.cuda.ExternalStream(pagani.lib().pg_stream(ctx.h))
    if args.case == "fw_batch":
        series = synth.roi_batch(args.graphs, ROI_N[0], ROI_N[1], ROI_T, N_SIG, synth.subject_seed(4))
        graphs = [ctx.build_graph(b, mode="r", value=ROI_R, sign="signed", weighted=True)[0] for b in series]
        call = lambda: ctx.fw_batched(graphs)  # noqa: E731
    else:
        bold = synth.bold_series(N_VOX, T_LEN, N_SIG, synth.subject_seed(2, 0))
        sp = 1.0 if args.case in ("gram", "brandes", "newman") else COHORT_SPARSITY
        g, _ = ctx.build_graph(bold, mode="s", value=sp, sign="abs")
        m = g.info[1] // 2
        if args.case == "paths":
            rg, _ = ctx.maslov(g, 7, COHORT_SWAPS * m)
            call = lambda: ctx.paths(rg)  # noqa: E731
        elif args.case == "maslov":
            call = lambda: ctx.maslov(g, 7, COHORT_SWAPS * m)[0].free()  # noqa: E731
        elif args.case == "gram":
            call = lambda: ctx.build_graph(bold, mode="s", value=1.0, sign="abs")[0].free()  # noqa: E731
        elif args.case == "newman":
            call = lambda: ctx.newman(g)  # noqa: E731
        else:
            call = lambda: ctx.betweenness(g)  # noqa: E731
    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    call()
    e1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "voxels": N_VOX, "ms": e0.elapsed_time(e1)}), flush=True)
    ctx.close()


# ------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32-leg", action="store_true")
    ap.add_argument("--no-cohort", action="store_true", help="skip the subject-average figure")
    ap.add_argument("--cohort-subjects", type=int, default=3,
                    help="subjects of the cohort configuration timed beside the step (0: skip)")
    ap.add_argument("--no-precision-report", action="store_true")
    ap.add_argument("--no-roi-batch", action="store_true", help="skip the 512-graph weighted batch figure")
    ap.add_argument("--case", default="step", choices=["step", "paths", "maslov", "fw_batch", "gram", "brandes", "newman"],
                    help="profiling aid: one small workload of one kernel family instead of the benchmark")
    ap.add_argument("--graphs", type=int, default=64, help="--case fw_batch: graphs in the batch")
    ap.add_argument("--voxels", type=int, default=N_VOX,
                    help="profiling aid: a smaller subject for ncu captures (the metric is quoted at 58000)")
    args = ap.parse_args()
    if args.gpus > 1 and "RANK" not in os.environ:
        spawn_ranks(args.gpus, run, args)   # started without torchrun
        return
    run(args)


def run(args):
    set_voxels(args.voxels)
    if args.case != "step":
        kernel_case(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    import pagani
    from pagani import synth

    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    ctx = pagani.Context(local)
    stream = torch.cuda.ExternalStream(pagani.lib().pg_stream(ctx.h))

    bold = synth.bold_series(N_VOX, T_LEN, N_SIG, rank_subject_seed(rank))
    bold_dev = torch.from_numpy(bold).to(f"cuda:{local}")
    bold_pin = torch.from_numpy(bold).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    hbm_peak, bf16_peak, peak_kind = _peaks()
    d2h_bytes = N_VOX * (4 + 4 + 8 + 4 + 4 + 4)   # degree, cp, tri, bc, eff, labels

    def subject(precision, on_device, timings=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        if on_device:
            g, info = ctx.build_graph(None, mode="s", value=SPARSITY, sign="abs", precision=precision,
                                      device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
        else:
            g, info = ctx.build_graph(bold_pin.numpy(), mode="s", value=SPARSITY, sign="abs", precision=precision)
        deg, iso = ctx.degree(g)
        cp, tri, cpm = ctx.clustering(g)
        ev[0].record(stream)
        bc, bc64, eff, lp = ctx.betweenness(g, with_paths=True)
        ev[1].record(stream)
        labels, Q, nmod = ctx.newman(g)
        ev[2].record(stream)
        if timings is not None:
            torch.cuda.synchronize()
            timings.append({"bc_ms": ev[0].elapsed_time(ev[1]), "newman_ms": ev[1].elapsed_time(ev[2]),
                            "build": info, "nnz": g.info[1], "lp": lp, "Q": Q, "modules": nmod,
                            "bc64": bc64, "labels": labels})
        g.free()

    def timed(precision, on_device, steps, warmup, timings=None, prof=None):
        if prof is not None:        # per-kernel events; the warm-up steps fill the event pool
            ctx.profile(True)
        for _ in range(warmup):
            subject(precision, on_device)
        if prof is not None:
            ctx.profile_reset()     # only the timed steps count
        ms = []
        for _ in range(steps):
            flush.fill_(1)          # evict L2 between timed steps
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            subject(precision, on_device, timings)
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            if world > 1:
                t = reduce_max_ms(t, f"cuda:{local}")
            ms.append(t)
        if prof is not None:
            for k in ("k_brandes", "k_bc_dense"):
                prof[k] = ctx.kernel_time(k)
            ctx.profile(False)
        return float(np.mean(ms)), ms

    launches0 = ctx.launches
    clocks = ClockSampler(local)
    clocks.start()
    timings = []
    kprof = {}
    ms_dev, all_ms = timed(args.precision, True, args.steps, args.warmup, timings, prof=kprof)
    clk = clocks.stop()
    launches = (ctx.launches - launches0) // max(1, args.steps + args.warmup)
    ms_e2e, _ = timed(args.precision, False, args.steps, 1)
    fp32 = None
    if not args.no_fp32_leg and args.precision != "fp32":
        ms_fp32, _ = timed("fp32", True, max(1, args.steps), 1)
        fp32 = {"value": world * 60000.0 / ms_fp32, "unit": "subjects/min", "ms_per_step": ms_fp32}

    # eigenvector centrality (the CUEC power method) on the same subject
    # graph, outside the timed step: CUDA events around the call, after one
    # warm-up call
    g_ec, _ = ctx.build_graph(None, mode="s", value=SPARSITY, sign="abs", precision=args.precision,
                              device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
    ctx.eigen_centrality(g_ec)
    ec_ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, ec_lam, ec_it, _ = ctx.eigen_centrality(g_ec)
        e1.record(stream)
        torch.cuda.synchronize()
        ec_ms.append(e0.elapsed_time(e1))
    ec_nnz = g_ec.info[1]
    g_ec.free()
    ec_t = float(np.median(ec_ms))
    eigen = {"ms": ec_t, "iterations": ec_it, "eigenvalue": ec_lam,
             "gteps": ec_nnz * ec_it / (ec_t / 1000.0) / 1e9}

    # subject averaging (CUCorMat to_average yf) on the same series: the FP64
    # Gram + Fisher accumulate of one subject, and the graph of the average
    # (top 1%), CUDA events around each call after one warm-up add
    cohort = None
    if not args.no_cohort:
        M1 = N_VOX * (N_VOX - 1) // 2
        with ctx.cohort(N_VOX, fisher=True) as c:
            c.add(device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
            add_ms = []
            for _ in range(2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                c.add(device_ptr=(bold_dev.data_ptr(), (T_LEN, N_VOX)))
                e1.record(stream)
                torch.cuda.synchronize()
                add_ms.append(e0.elapsed_time(e1))
            g_c, _ = c.graph("s", SPARSITY)           # keys allocated on first use
            g_c.free()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g_c, cinfo = c.graph("s", SPARSITY)
            e1.record(stream)
            torch.cuda.synchronize()
            g_c.free()
        add_t = float(np.median(add_ms))
        cohort = {"subjects": 3, "fisher": True, "ms_per_subject_add": add_t,
                  "fp64_gram_tflops": 2.0 * M1 * T_LEN / (add_t / 1000.0) / 1e12,
                  "flops_counted": "one FP64 fused multiply-add (2 flop) per pair and time point",
                  "ms_graph_top1pct": e0.elapsed_time(e1), "edges": cinfo["edges"]}

    value = world * 60000.0 / ms_dev
    e2e = world * 60000.0 / ms_e2e
    tm = timings[-1]
    prec_rep = None if args.no_precision_report else precision_report(ctx, bold_dev, tm)
    build = build_stage(ctx, bold_dev, stream, hbm_peak, bf16_peak)
    cohort5 = cohort_leg(ctx, args.cohort_subjects, rank) if args.cohort_subjects > 0 else None
    roi = None if args.no_roi_batch else roi_batch_leg(ctx, stream)
    nnz = tm["nnz"]
    # roofline of the dominant kernel, k_brandes (the gather sweeps of every
    # 128-source batch: level 1, the levels after the tensor-core ones and the
    # whole backward sweep), timed with CUDA events around its launches during
    # the timed steps.  Algorithmic bytes per batch: those of the backward
    # sweep alone -- per source nnz*4 col + (N+1)*4 rowptr + N*(4 dist +
    # 8 sigma + 8 delta) -- so the figure leaves out the forward levels the
    # kernel also runs (conservative).
    n_batches = (N_VOX + 127) // 128
    kb_launches, kb_ms = kprof["k_brandes"]
    kb_ms_batch = kb_ms / max(1, args.steps * n_batches)
    per_src_bwd = nnz * 4 + (N_VOX + 1) * 4 + N_VOX * (4 + 8 + 8)
    bytes_batch = per_src_bwd * 128
    achieved = bytes_batch / (kb_ms_batch / 1000.0) / 1e9 if kb_ms_batch > 0 else None
    bc_s = tm["bc_ms"] / 1000.0
    gteps = N_VOX * nnz / bc_s / 1e9
    # the tensor-core levels (k_bc_dense): one pass over the dense 0/1
    # adjacency per launch, HBM-bound
    kd_launches, kd_ms = kprof["k_bc_dense"]
    np_pad = (N_VOX + 127) // 128 * 128
    tensor_levels = None
    if kd_launches:
        kd_ms_launch = kd_ms / kd_launches
        tensor_levels = {"kernel": "k_bc_dense", "launches_per_step": kd_launches / args.steps,
                         "ms_per_launch": kd_ms_launch, "bytes_per_launch": np_pad * np_pad,
                         "achieved_gbs": np_pad * np_pad / (kd_ms_launch / 1000.0) / 1e9,
                         "frac": np_pad * np_pad / (kd_ms_launch / 1000.0) / 1e9 / hbm_peak,
                         "ms_per_step": kd_ms / args.steps}
    line = {
        "metric": "cohort subjects/min @58k voxels", "value": value, "unit": "subjects/min",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_dev,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16" if args.precision == "bf16x3" else "fp32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": args.precision, "global_batch": world,
                   "parallelism": f"replicas{world}", "l2": "flushed (256 MB write) before every timed step",
                   "edges": nnz // 2, "tau": tm["build"]["tau"]},
        "e2e": {"value": e2e, "unit": "subjects/min", "h2d_bytes_per_step": N_VOX * T_LEN * 4,
                "d2h_bytes_per_step": d2h_bytes},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_brandes", "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak if achieved else None,
                     "traffic": BRANDES_DRAM_BYTES_PER_BATCH_58K if N_VOX == 58000 else None,
                     "traffic_source": "ncu one-pass dram__bytes_read.sum + dram__bytes_write.sum of the k_brandes "
                                       "launches of one batch at 58k (profiles/k_brandes_subject58k.md)",
                     "bound_note": "the DRAM traffic is 0.065 of the algorithmic bytes: batching shares every "
                                   "CSR read among 128 sources and the per-node state is served by L2; ncu on the "
                                   "16k subject (profiles/k_brandes_subject16k.md) shows L2 hit rate 92.2 %, L2 "
                                   "throughput 18.1 %, issue active 39.2 % and long-scoreboard then barrier stalls "
                                   "on top -- L2 latency and the level barriers bound the sweep, not HBM",
                     "algorithmic_bytes_per_launch": bytes_batch,
                     "per_launch": "one 128-source batch (its k_brandes launches); algorithmic bytes of the "
                                   "backward sweep only",
                     "ms_per_batch": kb_ms_batch, "launches_per_step": kb_launches / args.steps,
                     "peak_source": peak_kind},
        "tensor_levels": tensor_levels,
        "bc_gteps": gteps, "bc_mteps_reference_formula": nnz * N_VOX / (tm["bc_ms"]) / 1024 ** 2,
        "stage_ms": {"build": {k: tm["build"][k] for k in ("ms_zscore", "ms_hist", "ms_emit", "ms_select", "ms_csr")},
                     "betweenness_and_paths": tm["bc_ms"], "newman": tm["newman_ms"]},
        "step_ms_all": all_ms,
        "eigen_centrality": eigen,
        "subject_average": cohort,
        "precision_report": prec_rep,
        "build_stage": build,
        "cohort": cohort5,
        "roi_batch": roi,
        "clocks": clk,
    }
    if fp32:
        line["fp32_path"] = fp32
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
