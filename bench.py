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


def _cpu_baseline(n_sample=4000, threads=None):
    """The reference's own CPU pipeline (oracle/_ref) on a down-scaled subject.

    The reference CPU code cannot run the 58k subject in bounded time
    (single-thread Brandes alone is hours; CorMat_cpu_MT overflows its int
    pair index beyond ~18.5k voxels).  The sample is a complete subject with
    the same generator, T and density at n_sample voxels; each stage's time
    is scaled to N = 58,000 by its work: N^2 for the correlation, selection
    and CSR build, N^3 (fixed density, so N * nnz) for clustering, BFS path
    length, betweenness and modularity.
    """
    from oracle import oracle as O
    from pagani import synth
    threads = threads or os.cpu_count() or 1
    os.environ["PAGANI_REF_THREADS"] = str(threads)
    ref = O.Ref()
    bold = synth.bold_series(n_sample, T_LEN, N_SIG, synth.subject_seed(2, 99))
    st = {}
    t = time.perf_counter()
    cm = ref.cormat_cpu_mt(bold, threads)
    st["correlation"] = time.perf_counter() - t
    k = O.sparsity_k(n_sample, SPARSITY)
    t = time.perf_counter()
    R, C, _ = ref.graph_s(np.abs(cm), n_sample, k)
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
    scale2 = (N_VOX / n_sample) ** 2
    scale3 = (N_VOX / n_sample) ** 3
    sec = (st["correlation"] + st["threshold_csr"]) * scale2 + \
        (st["cp"] + st["paths"] + st["betweenness"] + st["newman"]) * scale3
    return {
        "value": 60.0 / sec, "unit": "subjects/min", "cores": threads, "kind": "reference",
        "sample": f"reference CPU pipeline (CorMat_cpu_MT, FormFullGraph_s on |r|, FormCSRGraph, Cp, APSP_BFS, "
                  f"Betweenness_CPU, Partition) on a complete N={n_sample} subject, T={T_LEN}, top 1%; stage "
                  f"times scaled to N={N_VOX} by N^2 (correlation/threshold) and N^3 (graph metrics); "
                  f"measured sample seconds " + json.dumps({k2: round(v, 3) for k2, v in st.items()}),
        "extrapolated_seconds_per_subject": sec,
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
    ap.add_argument("--voxels", type=int, default=N_VOX,
                    help="profiling aid: a smaller subject for ncu captures (the metric is quoted at 58000)")
    args = ap.parse_args()
    if args.gpus > 1 and "RANK" not in os.environ:
        spawn_ranks(args.gpus, run, args)   # started without torchrun
        return
    run(args)


def run(args):
    set_voxels(args.voxels)
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
                            "build": info, "nnz": g.info[1], "lp": lp, "Q": Q, "modules": nmod})
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
