"""Python front end of libpagani (ctypes over the C ABI in include/pagani.h).

The compute lives in libpagani.so (hand-written sm_100a kernels).  There is no
CPU fallback: importing works anywhere, but every call that computes needs the
library and a B200; a missing library raises immediately.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libpagani.so")

PG_THRESH_R, PG_THRESH_SPARSITY = 0, 1
PG_SIGNED, PG_ABS = 0, 1
PG_FP32, PG_SPLIT_BF16 = 0, 1

_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
           4: "too large", 5: "internal check failed", 6: "timeout", 7: "no usable sm_100 device"}

# Every entry point the header declares (kept in step with include/pagani.h).
EXPORTS = [
    "pg_create", "pg_destroy", "pg_last_error", "pg_status_string", "pg_synchronize", "pg_stream",
    "pg_launch_count", "pg_graph_from_csr", "pg_graph_info", "pg_graph_to_csr", "pg_graph_free",
    "pg_build_opts_default", "pg_build_graph", "pg_sparsity_edges", "pg_correlation_packed",
    "pg_degree", "pg_clustering", "pg_paths", "pg_betweenness", "pg_bfs_sigma", "pg_fw_paths",
    "pg_fw_batched", "pg_newman", "pg_newman_weighted", "pg_eigen_centrality", "pg_participation", "pg_maslov", "pg_maslov_round_size", "pg_smallworld",
    "pg_clustering_noalloc", "pg_clustering_noalloc_max_nodes",
    "pg_cohort_create", "pg_cohort_add", "pg_cohort_graph", "pg_cohort_packed", "pg_cohort_info",
    "pg_cohort_free", "pg_profile_enable", "pg_profile_reset", "pg_profile_get",
    "pg_run_opts_default", "pg_surrogate_seed", "pg_run_subjects", "pg_debug_stall_next_gram",
]


def build() -> None:
    subprocess.run(["make", "-s", "-j8", "-C", PKG_DIR], check=True)


class PaganiError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


class BuildOpts(ct.Structure):
    _fields_ = [("mode", ct.c_int32), ("value", ct.c_double), ("sign", ct.c_int32),
                ("precision", ct.c_int32), ("weighted", ct.c_int32), ("guard", ct.c_double),
                ("input_on_device", ct.c_int32), ("exact_weights", ct.c_int32)]


class BuildInfo(ct.Structure):
    _fields_ = [("tau", ct.c_double), ("edges", ct.c_int64), ("band_pairs", ct.c_int64),
                ("above_pairs", ct.c_int64), ("zero_variance", ct.c_int32),
                ("sparsity_percent", ct.c_double), ("ms_zscore", ct.c_double), ("ms_hist", ct.c_double),
                ("ms_emit", ct.c_double), ("ms_select", ct.c_double), ("ms_csr", ct.c_double),
                ("band_err_max", ct.c_double), ("band_err_mean", ct.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Subject(ct.Structure):
    _fields_ = [("bold", ct.c_void_p), ("N", ct.c_int32), ("T", ct.c_int32), ("degree", ct.c_void_p),
                ("cp", ct.c_void_p), ("eff", ct.c_void_p), ("bc", ct.c_void_p), ("modules", ct.c_void_p),
                ("edges", ct.c_int64), ("tau", ct.c_double), ("cp_mean", ct.c_double), ("lp", ct.c_double),
                ("Q", ct.c_double), ("n_modules", ct.c_int32), ("gamma", ct.c_double), ("lambda_", ct.c_double),
                ("sigma", ct.c_double), ("surrogate_graph_replays", ct.c_int32)]


class RunOpts(ct.Structure):
    _fields_ = [("build", BuildOpts), ("n_random", ct.c_int32), ("swaps_per_edge", ct.c_int64),
                ("seed", ct.c_uint64), ("cuda_graphs", ct.c_int32)]


LOG_FN = ct.CFUNCTYPE(None, ct.c_char_p, ct.c_void_p)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = ct.CDLL(LIB_PATH)
        vp, i32, i64, dbl = ct.c_void_p, ct.c_int32, ct.c_int64, ct.c_double
        P = ct.POINTER
        L.pg_create.argtypes = [P(vp), ct.c_int]
        L.pg_destroy.argtypes = [vp]
        L.pg_last_error.argtypes = [vp]
        L.pg_last_error.restype = ct.c_char_p
        L.pg_status_string.argtypes = [ct.c_int]
        L.pg_status_string.restype = ct.c_char_p
        L.pg_synchronize.argtypes = [vp]
        L.pg_stream.argtypes = [vp]
        L.pg_stream.restype = vp
        L.pg_launch_count.argtypes = [vp]
        L.pg_launch_count.restype = i64
        L.pg_graph_from_csr.argtypes = [vp, vp, vp, vp, i32, i64, i32, P(vp)]
        L.pg_graph_info.argtypes = [vp, P(i32), P(i64), P(i32)]
        L.pg_graph_to_csr.argtypes = [vp, vp, vp, vp, vp, i32]
        L.pg_graph_free.argtypes = [vp]
        L.pg_build_opts_default.argtypes = [P(BuildOpts)]
        L.pg_build_opts_default.restype = None
        L.pg_build_graph.argtypes = [vp, vp, i32, i32, P(BuildOpts), P(vp), P(BuildInfo)]
        L.pg_sparsity_edges.argtypes = [i32, ct.c_float]
        L.pg_sparsity_edges.restype = i64
        L.pg_correlation_packed.argtypes = [vp, vp, i32, i32, i32, i32, vp]
        L.pg_degree.argtypes = [vp, vp, vp, P(i32)]
        L.pg_clustering.argtypes = [vp, vp, i32, i32, vp, vp, P(dbl)]
        L.pg_paths.argtypes = [vp, vp, vp, vp, P(dbl), vp, i32, P(i32)]
        L.pg_betweenness.argtypes = [vp, vp, vp, vp, vp, P(dbl)]
        L.pg_bfs_sigma.argtypes = [vp, vp, vp, i32, vp, vp]
        L.pg_fw_paths.argtypes = [vp, vp, vp, vp, P(dbl)]
        L.pg_fw_batched.argtypes = [vp, P(vp), i32, vp, vp, vp, vp]
        L.pg_newman.argtypes = [vp, vp, i32, vp, P(dbl), P(i32), LOG_FN, vp]
        L.pg_newman_weighted.argtypes = [vp, vp, vp, i32, vp, P(dbl), P(i32), LOG_FN, vp]
        L.pg_eigen_centrality.argtypes = [vp, vp, i32, vp, P(dbl), P(i32), P(dbl)]
        L.pg_participation.argtypes = [vp, vp, vp, vp, vp, P(i32)]
        L.pg_maslov.argtypes = [vp, vp, ct.c_uint64, i64, P(vp), P(i64)]
        L.pg_maslov_round_size.argtypes = [i64]
        L.pg_maslov_round_size.restype = i64
        L.pg_smallworld.argtypes = [dbl, vp, i32, dbl, vp, i32, P(dbl), P(dbl), P(dbl)]
        L.pg_clustering_noalloc.argtypes = [vp, vp, i32, vp, vp, vp]
        L.pg_clustering_noalloc_max_nodes.argtypes = []
        L.pg_clustering_noalloc_max_nodes.restype = i64
        L.pg_cohort_create.argtypes = [vp, i32, i32, i32, P(vp)]
        L.pg_cohort_add.argtypes = [vp, vp, vp, i32, i32]
        L.pg_cohort_graph.argtypes = [vp, vp, i32, dbl, P(vp), P(BuildInfo)]
        L.pg_cohort_packed.argtypes = [vp, vp, vp]
        L.pg_cohort_info.argtypes = [vp, P(i32), P(i32)]
        L.pg_cohort_free.argtypes = [vp]
        L.pg_profile_enable.argtypes = [vp, i32]
        L.pg_profile_reset.argtypes = [vp]
        L.pg_profile_get.argtypes = [vp, ct.c_char_p, P(i64), P(dbl)]
        L.pg_run_opts_default.argtypes = [P(RunOpts)]
        L.pg_run_opts_default.restype = None
        L.pg_surrogate_seed.argtypes = [ct.c_uint64, i32, i32]
        L.pg_surrogate_seed.restype = ct.c_uint64
        L.pg_run_subjects.argtypes = [vp, P(Subject), i32, P(RunOpts)]
        L.pg_debug_stall_next_gram.argtypes = [vp, ct.c_uint64]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ct.c_void_p(a.ctypes.data)


def sparsity_edges(N, s_percent):
    return int(lib().pg_sparsity_edges(N, s_percent))


def maslov_round_size(M):
    return int(lib().pg_maslov_round_size(M))


class Graph:
    """Device-resident CSR graph owned by a Context."""

    def __init__(self, ctx, handle):
        self.ctx, self.h = ctx, handle   # the reference keeps the context alive

    @property
    def info(self):
        n, nnz, w = ct.c_int32(), ct.c_int64(), ct.c_int32()
        lib().pg_graph_info(self.h, ct.byref(n), ct.byref(nnz), ct.byref(w))
        return n.value, nnz.value, bool(w.value)

    def to_csr(self):
        n, nnz, w = self.info
        R = np.empty(n + 1, np.int32)
        C = np.empty(max(nnz, 1), np.int32)
        V = np.empty(max(nnz, 1), np.float32) if w else None
        self.ctx._check(lib().pg_graph_to_csr(self.ctx.h, self.h, _p(R), _p(C), _p(V), 0))
        return R, C[:nnz], (V[:nnz] if w else None)

    def free(self):
        if self.h:
            lib().pg_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Cohort:
    """Subject-averaged correlation (CUCorMat's to_average modes) held on the
    device: add() subjects, then graph() or packed()."""

    def __init__(self, ctx, N, fisher=False, weighted=False):
        self.ctx, self.N, self.weighted = ctx, N, weighted
        h = ct.c_void_p()
        ctx._check(lib().pg_cohort_create(ctx.h, N, int(fisher), int(weighted), ct.byref(h)))
        self.h = h

    def add(self, bold_TxN=None, device_ptr=None):
        """One subject: (T, N) float32 on the host, or device_ptr = (ptr, (T, N))."""
        if device_ptr is not None:
            ptr, (T, N) = device_ptr
            src, on_dev = ct.c_void_p(ptr), 1
        else:
            bold = np.ascontiguousarray(bold_TxN, np.float32)
            T, N = bold.shape
            src, on_dev = _p(bold), 0
        if N != self.N:
            raise ValueError(f"subject has {N} voxels, cohort has {self.N}")
        self.ctx._check(lib().pg_cohort_add(self.ctx.h, self.h, src, T, on_dev))

    @property
    def subjects(self):
        n, s = ct.c_int32(), ct.c_int32()
        lib().pg_cohort_info(self.h, ct.byref(n), ct.byref(s))
        return s.value

    def graph(self, mode="r", value=0.3):
        info = BuildInfo()
        h = ct.c_void_p()
        m = PG_THRESH_SPARSITY if mode in ("s", "sparsity") else PG_THRESH_R
        self.ctx._check(lib().pg_cohort_graph(self.ctx.h, self.h, m, value, ct.byref(h), ct.byref(info)))
        return Graph(self.ctx, h), info.as_dict()

    def packed(self):
        M1 = self.N * (self.N - 1) // 2
        out = np.empty(max(M1, 1), np.float32)
        self.ctx._check(lib().pg_cohort_packed(self.ctx.h, self.h, _p(out)))
        return out[:M1]

    def free(self):
        if self.h:
            lib().pg_cohort_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()


class Context:
    def __init__(self, device=0):
        h = ct.c_void_p()
        st = lib().pg_create(ct.byref(h), device)
        if st != 0:
            raise PaganiError(st, "pg_create failed")
        self.h = h

    def close(self):
        if self.h:
            lib().pg_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != 0:
            raise PaganiError(st, lib().pg_last_error(self.h).decode())

    @property
    def launches(self):
        return int(lib().pg_launch_count(self.h))

    def profile(self, on=True):
        """Per-kernel event timing on (or off); see kernel_time()."""
        self._check(lib().pg_profile_enable(self.h, int(on)))

    def profile_reset(self):
        self._check(lib().pg_profile_reset(self.h))

    def kernel_time(self, name):
        """(launches, summed ms) of one profiled kernel since the last reset."""
        n, ms = ct.c_int64(), ct.c_double()
        self._check(lib().pg_profile_get(self.h, name.encode(), ct.byref(n), ct.byref(ms)))
        return n.value, ms.value

    def synchronize(self):
        self._check(lib().pg_synchronize(self.h))

    # -------------------------------------------------------------- graphs
    def graph(self, R, C, V=None):
        R = np.ascontiguousarray(R, np.int32)
        C = np.ascontiguousarray(C, np.int32)
        V = None if V is None else np.ascontiguousarray(V, np.float32)
        h = ct.c_void_p()
        self._check(lib().pg_graph_from_csr(self.h, _p(R), _p(C), _p(V), len(R) - 1, len(C), 0,
                                            ct.byref(h)))
        return Graph(self, h)

    def build_graph(self, bold_TxN, mode="r", value=0.3, sign="signed", precision="bf16x3",
                    weighted=False, guard=2e-3, exact_weights=True, device_ptr=None):
        """Network construction; bold is (T, N) float32 (or device_ptr with shape)."""
        o = BuildOpts()
        lib().pg_build_opts_default(ct.byref(o))
        o.mode = PG_THRESH_SPARSITY if mode in ("s", "sparsity") else PG_THRESH_R
        o.value = value
        o.sign = PG_ABS if sign == "abs" else PG_SIGNED
        o.precision = PG_FP32 if precision == "fp32" else PG_SPLIT_BF16
        o.weighted = int(weighted)
        o.guard = guard
        o.exact_weights = int(exact_weights)
        info = BuildInfo()
        h = ct.c_void_p()
        if device_ptr is not None:
            ptr, (T, N) = device_ptr
            o.input_on_device = 1
            self._check(lib().pg_build_graph(self.h, ct.c_void_p(ptr), N, T, ct.byref(o), ct.byref(h),
                                             ct.byref(info)))
        else:
            bold = np.ascontiguousarray(bold_TxN, np.float32)
            T, N = bold.shape
            self._check(lib().pg_build_graph(self.h, _p(bold), N, T, ct.byref(o), ct.byref(h), ct.byref(info)))
        return Graph(self, h), info.as_dict()

    def correlation_packed(self, bold_TxN, weighted=False):
        bold = np.ascontiguousarray(bold_TxN, np.float32)
        T, N = bold.shape
        out = np.empty(max(N * (N - 1) // 2, 1), np.float32)
        self._check(lib().pg_correlation_packed(self.h, _p(bold), N, T, int(weighted), 0, _p(out)))
        return out[: N * (N - 1) // 2]

    def cohort(self, N, fisher=False, weighted=False):
        """Subject averaging (CUCorMat to_average yn/yf): a Cohort of N voxels."""
        return Cohort(self, N, fisher, weighted)

    def run_subjects(self, bolds, mode="s", value=1.0, sign="abs", n_random=0, swaps_per_edge=2, seed=1,
                     metrics=("degree", "cp", "eff", "bc", "modules"), weighted=False, precision="bf16x3",
                     cuda_graphs=True, device_ptrs=None):
        """pg_run_subjects over (T, N) float32 series: one dict per subject with
        the requested per-node arrays and the scalar results.  device_ptrs:
        optional list of (pointer, (T, N)) of series already on the device."""
        o = RunOpts()
        lib().pg_run_opts_default(ct.byref(o))
        o.build.mode = PG_THRESH_SPARSITY if mode in ("s", "sparsity") else PG_THRESH_R
        o.build.value = value
        o.build.sign = PG_ABS if sign == "abs" else PG_SIGNED
        o.build.weighted = int(weighted)
        o.build.precision = PG_FP32 if precision == "fp32" else PG_SPLIT_BF16
        o.build.input_on_device = int(device_ptrs is not None)
        o.n_random, o.swaps_per_edge, o.seed = n_random, swaps_per_edge, seed
        o.cuda_graphs = int(cuda_graphs)
        count = len(device_ptrs) if device_ptrs is not None else len(bolds)
        keep, subs = [], (Subject * max(1, count))()
        outs = []
        for k in range(count):
            if device_ptrs is not None:
                ptr, (T, N) = device_ptrs[k]
            else:
                b = np.ascontiguousarray(bolds[k], np.float32)
                T, N = b.shape
                keep.append(b)
                ptr = b.ctypes.data
            arrs = {m: np.zeros(N, np.int32 if m == "modules" else np.float32) for m in metrics}
            keep += list(arrs.values())
            subs[k].bold, subs[k].N, subs[k].T = ptr, N, T
            for m, a in arrs.items():
                setattr(subs[k], m, a.ctypes.data)
            outs.append(arrs)
        self._check(lib().pg_run_subjects(self.h, subs, count, ct.byref(o)))
        res = []
        for k, arrs in enumerate(outs):
            d = dict(arrs)
            for f in ("edges", "tau", "cp_mean", "lp", "Q", "n_modules", "gamma", "lambda_", "sigma",
                      "surrogate_graph_replays"):
                d[f.rstrip("_")] = getattr(subs[k], f)
            res.append(d)
        return res

    # ------------------------------------------------------------- metrics
    def degree(self, g):
        n = g.info[0]
        deg = np.empty(n, np.float32)
        iso = ct.c_int32()
        self._check(lib().pg_degree(self.h, g.h, _p(deg), ct.byref(iso)))
        return deg, iso.value

    def clustering(self, g, kind="binary", vmax_first_n=False):
        n = g.info[0]
        cp = np.empty(n, np.float32)
        tri = np.empty(n, np.int64) if kind == "binary" else None
        mean = ct.c_double()
        self._check(lib().pg_clustering(self.h, g.h, 0 if kind == "binary" else 1, int(vmax_first_n),
                                        _p(cp), _p(tri), ct.byref(mean)))
        return cp, tri, mean.value

    def paths(self, g, max_hop=64):
        n = g.info[0]
        eff = np.empty(n, np.float32)
        inv = np.empty(n, np.float64)
        hist = np.zeros(max_hop + 1, np.int64)
        lp = ct.c_double()
        diam = ct.c_int32()
        self._check(lib().pg_paths(self.h, g.h, _p(eff), _p(inv), ct.byref(lp), _p(hist), max_hop,
                                   ct.byref(diam)))
        return eff, inv, lp.value, hist, diam.value

    def betweenness(self, g, with_paths=False):
        n = g.info[0]
        bc = np.empty(n, np.float32)
        bc64 = np.empty(n, np.float64)
        eff = np.empty(n, np.float32) if with_paths else None
        lp = ct.c_double()
        self._check(lib().pg_betweenness(self.h, g.h, _p(bc), _p(bc64), _p(eff),
                                         ct.byref(lp) if with_paths else None))
        return (bc, bc64, eff, lp.value) if with_paths else (bc, bc64)

    def bfs_sigma(self, g, sources):
        n = g.info[0]
        src = np.ascontiguousarray(sources, np.int32)
        dist = np.empty((len(src), n), np.int32)
        sigma = np.empty((len(src), n), np.int64)
        self._check(lib().pg_bfs_sigma(self.h, g.h, _p(src), len(src), _p(dist), _p(sigma)))
        return dist, sigma

    def fw_paths(self, g, want_dist=False):
        n = g.info[0]
        dist = np.empty((n, n), np.float32) if want_dist else None
        eff = np.empty(n, np.float32)
        lp = ct.c_double()
        self._check(lib().pg_fw_paths(self.h, g.h, _p(dist), _p(eff), ct.byref(lp)))
        return (eff, lp.value, dist) if want_dist else (eff, lp.value)

    def fw_batched(self, graphs):
        sizes = [g.info[0] for g in graphs]
        tot = int(sum(sizes))
        eff = np.empty(max(tot, 1), np.float32)
        cp = np.empty(max(tot, 1), np.float32)
        lp = np.empty(len(graphs), np.float64)
        cpm = np.empty(len(graphs), np.float64)
        arr = (ct.c_void_p * len(graphs))(*[g.h.value for g in graphs])
        self._check(lib().pg_fw_batched(self.h, arr, len(graphs), _p(eff), _p(lp), _p(cp), _p(cpm)))
        out, o = [], 0
        for gi, n in enumerate(sizes):
            out.append((eff[o:o + n].copy(), lp[gi], cp[o:o + n].copy(), cpm[gi]))
            o += n
        return out

    def newman(self, g, gpu_rule_above=25000, log=None):
        n = g.info[0]
        labels = np.empty(n, np.int32)
        Q = ct.c_double()
        nm = ct.c_int32()
        lines = []

        def _cb(line, _u):
            lines.append(line.decode())

        cb = LOG_FN(_cb)
        self._check(lib().pg_newman(self.h, g.h, gpu_rule_above, _p(labels), ct.byref(Q), ct.byref(nm), cb, None))
        if log is not None:
            log.extend(lines)
        return labels, Q.value, nm.value

    def newman_weighted(self, g, weights_of=None, gpu_rule_above=25000, log=None):
        """The weighted Newman tool's partition (pg_newman_weighted); weights_of
        is the graph whose value array is read by position (default g)."""
        n = g.info[0]
        labels = np.empty(n, np.int32)
        Q = ct.c_double()
        nm = ct.c_int32()
        lines = []

        def _cb(line, _u):
            lines.append(line.decode())

        cb = LOG_FN(_cb)
        w = None if weights_of is None else weights_of.h
        self._check(lib().pg_newman_weighted(self.h, g.h, w, gpu_rule_above, _p(labels), ct.byref(Q), ct.byref(nm),
                                             cb, None))
        if log is not None:
            log.extend(lines)
        return labels, Q.value, nm.value

    def eigen_centrality(self, g, raw=False):
        """Eigenvector centrality (pg_eigen_centrality): returns (ec float64[n],
        eigenvalue, iterations, residual).  raw=True gives y = A x of the last
        step (the weighted CUEC tool's output), else the normalised x."""
        n = g.info[0]
        ec = np.empty(max(n, 1), np.float64)
        lam, res = ct.c_double(), ct.c_double()
        it = ct.c_int32()
        self._check(lib().pg_eigen_centrality(self.h, g.h, int(bool(raw)), _p(ec), ct.byref(lam), ct.byref(it),
                                              ct.byref(res)))
        return ec[:n], lam.value, it.value, res.value

    def participation(self, g, module):
        """Participation coefficient (pg_participation): module = float labels
        1..K per node; returns (pc, pc_normalised, K), float32."""
        n = g.info[0]
        mod = np.ascontiguousarray(module, np.float32)
        pc = np.empty(max(n, 1), np.float32)
        pn = np.empty(max(n, 1), np.float32)
        K = ct.c_int32()
        self._check(lib().pg_participation(self.h, g.h, _p(mod), _p(pc), _p(pn), ct.byref(K)))
        return pc[:n], pn[:n], K.value

    def maslov(self, g, seed, attempts):
        h = ct.c_void_p()
        c = ct.c_int64()
        self._check(lib().pg_maslov(self.h, g.h, seed, attempts, ct.byref(h), ct.byref(c)))
        return Graph(self, h), c.value


def smallworld(cp, cp_rand, lp, lp_rand):
    cr = np.ascontiguousarray(cp_rand, np.float64)
    lr = np.ascontiguousarray(lp_rand, np.float64)
    g, l, s = ct.c_double(), ct.c_double(), ct.c_double()
    lib().pg_smallworld(cp, _p(cr), len(cr), lp, _p(lr), len(lr), ct.byref(g), ct.byref(l), ct.byref(s))
    return g.value, l.value, s.value
