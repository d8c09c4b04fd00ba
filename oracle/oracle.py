"""ctypes front end of the test checker.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the product library.

* ``liboracle.so``  -- the C restatement in oracle.c (FP64 conventions in its
  header).
* ``_ref/libref_*.so`` -- the reference's own CPU functions compiled from its
  sources (oracle/Makefile), used to pin the restatement.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = ct.c_void_p


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (and the reference groups when the tree exists)."""
    targets = ["all"]
    # the reference checkout: PAGANI_REF_ROOT, else a "reference" directory
    # beside the repository
    ref_root = os.environ.get("PAGANI_REF_ROOT", os.path.join(os.path.dirname(HERE), "..", "reference"))
    ref_root = os.path.abspath(ref_root)
    if ref is None:
        ref = os.path.isdir(ref_root)
    if ref:
        targets.append("ref")
    targets.append("big")
    subprocess.run(["make", "-s", "-C", HERE, f"REF_ROOT={ref_root}", *targets], check=True)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run oracle.build())")
    return ct.CDLL(path)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(os.path.join(HERE, "liboracle.so")):
            build(ref=False)
        L = _load(os.path.join(HERE, "liboracle.so"))
        L.or_zscore.argtypes = [_f32p, ct.c_int, ct.c_int, _f64p]
        L.or_zscore.restype = ct.c_int
        L.or_pair_r.argtypes = [_f64p, ct.c_int, ct.c_int, ct.c_int, ct.c_int]
        L.or_pair_r.restype = ct.c_double
        L.or_corr_packed.argtypes = [_f64p, ct.c_int, ct.c_int, ct.c_int, _f64p]
        L.or_sparsity_k.argtypes = [ct.c_int, ct.c_float]
        L.or_sparsity_k.restype = ct.c_int64
        L.or_weighted_r_threshold.argtypes = [ct.c_float]
        L.or_weighted_r_threshold.restype = ct.c_float
        L.or_graph_r.argtypes = [_f64p, ct.c_int, ct.c_double, ct.c_int, _i32p, _i32p, _vp, ct.c_int64]
        L.or_graph_r.restype = ct.c_int64
        L.or_graph_k.argtypes = [_f64p, ct.c_int, ct.c_int64, ct.c_int, ct.POINTER(ct.c_double),
                                 _i32p, _i32p, _vp, ct.c_int64]
        L.or_graph_k.restype = ct.c_int64
        L.or_degree.argtypes = [_i32p, _vp, ct.c_int, _f32p, ct.POINTER(ct.c_int32)]
        L.or_cp_binary.argtypes = [_i32p, _i32p, ct.c_int, _i64p, _f32p, ct.POINTER(ct.c_double)]
        L.or_onnela.argtypes = [_i32p, _i32p, _f32p, ct.c_int, ct.c_int, _f32p, ct.POINTER(ct.c_double)]
        L.or_bfs_paths.argtypes = [_i32p, _i32p, ct.c_int, _f64p, _i64p, ct.c_int, ct.POINTER(ct.c_double)]
        L.or_bfs_paths.restype = ct.c_int
        L.or_bfs_source.argtypes = [_i32p, _i32p, ct.c_int, ct.c_int, _i32p, _i64p]
        L.or_bfs_source.restype = ct.c_int
        L.or_brandes.argtypes = [_i32p, _i32p, ct.c_int, _f64p]
        L.or_fw_dense.argtypes = [_f32p, ct.c_int]
        L.or_weighted_paths.argtypes = [_i32p, _i32p, _f32p, ct.c_int, _f32p, ct.POINTER(ct.c_double)]
        L.or_weighted_paths.restype = ct.c_int
        L.or_newman.argtypes = [_i32p, _i32p, ct.c_int, ct.c_int, _i32p, ct.POINTER(ct.c_double),
                                ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]
        L.or_newman.restype = ct.c_int
        L.or_maslov.argtypes = [_i32p, _i32p, _vp, ct.c_int, ct.c_uint64, ct.c_int64, _i32p, _i32p, _vp]
        L.or_maslov.restype = ct.c_int64
        L.or_rewire_seq.argtypes = [_i32p, _i32p, _vp, ct.c_int, ct.c_uint32, ct.c_int64, _i32p, _i32p, _vp]
        L.or_rewire_seq.restype = ct.c_int64
        L.or_maslov_round_size.argtypes = [ct.c_int64]
        L.or_maslov_round_size.restype = ct.c_int64
        L.or_eigen_centrality.argtypes = [_i32p, _i32p, _vp, ct.c_int, ct.c_int, _f64p,
                                          ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)]
        L.or_eigen_centrality.restype = ct.c_int
        L.or_participation.argtypes = [_i32p, _i32p, _vp, ct.c_int, _f32p, _f32p, _f32p]
        L.or_participation.restype = ct.c_int
        L.or_newman_weighted.argtypes = [_i32p, _i32p, _f32p, ct.c_int64, ct.c_int, ct.c_int, _i32p,
                                         ct.POINTER(ct.c_double), ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]
        L.or_newman_weighted.restype = ct.c_int
        for f in ("or_ln", "or_exp", "or_fisher", "or_inv_fisher"):
            getattr(L, f).argtypes = [ct.c_double]
            getattr(L, f).restype = ct.c_double
        L.or_cohort_add.argtypes = [_f64p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, _f64p]
        L.or_cohort_finish.argtypes = [_f64p, ct.c_int64, ct.c_int, ct.c_int, _f64p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


# ----------------------------------------------------------------- restatement
def zscore(bold_TxN: np.ndarray):
    bold = np.ascontiguousarray(bold_TxN, dtype=np.float32)
    T, N = bold.shape
    z = np.empty((N, T), np.float64)
    nz = lib().or_zscore(bold, N, T, z)
    return z, nz


def pair_r(z, i, j, weighted=False):
    return lib().or_pair_r(z, z.shape[1], i, j, int(weighted))


def corr_packed(z, weighted=False):
    N, T = z.shape
    r = np.empty(N * (N - 1) // 2, np.float64)
    lib().or_corr_packed(np.ascontiguousarray(z), N, T, int(weighted), r)
    return r


def sparsity_k(N, s_percent):
    return int(lib().or_sparsity_k(N, s_percent))


def weighted_r_threshold(thr):
    return float(lib().or_weighted_r_threshold(thr))


def graph_r(r_packed, N, thr, abs_mode=False, weighted=False):
    M1 = N * (N - 1) // 2
    cap = 2 * M1
    R = np.zeros(N + 1, np.int32)
    C = np.zeros(max(cap, 1), np.int32)
    V = np.zeros(max(cap, 1), np.float32) if weighted else None
    nnz = lib().or_graph_r(r_packed, N, thr, int(abs_mode), R, C, _ptr(V), cap)
    return R, C[:nnz].copy(), (V[:nnz].copy() if weighted else None)


def graph_k(r_packed, N, k, abs_mode=False, weighted=False):
    M1 = N * (N - 1) // 2
    cap = 2 * M1
    R = np.zeros(N + 1, np.int32)
    C = np.zeros(max(cap, 1), np.int32)
    V = np.zeros(max(cap, 1), np.float32) if weighted else None
    tau = ct.c_double()
    nnz = lib().or_graph_k(r_packed, N, k, int(abs_mode), ct.byref(tau), R, C, _ptr(V), cap)
    return R, C[:nnz].copy(), (V[:nnz].copy() if weighted else None), tau.value


def degree(R, V=None):
    N = len(R) - 1
    deg = np.empty(N, np.float32)
    iso = ct.c_int32()
    lib().or_degree(R, _ptr(V), N, deg, ct.byref(iso))
    return deg, iso.value


def cp_binary(R, C):
    N = len(R) - 1
    tri = np.empty(N, np.int64)
    cp = np.empty(N, np.float32)
    mean = ct.c_double()
    lib().or_cp_binary(R, C, N, tri, cp, ct.byref(mean))
    return tri, cp, mean.value


def onnela(R, C, V, vmax_first_n=False):
    N = len(R) - 1
    cp = np.empty(N, np.float32)
    mean = ct.c_double()
    lib().or_onnela(R, C, V, N, int(vmax_first_n), cp, ct.byref(mean))
    return cp, mean.value


def bfs_paths(R, C, max_hop=64):
    N = len(R) - 1
    inv = np.empty(N, np.float64)
    hist = np.zeros(max_hop + 1, np.int64)
    lp = ct.c_double()
    dmax = lib().or_bfs_paths(R, C, N, inv, hist, max_hop, ct.byref(lp))
    return inv, hist, lp.value, dmax


def bfs_source(R, C, s):
    N = len(R) - 1
    dist = np.empty(N, np.int32)
    sigma = np.empty(N, np.int64)
    lib().or_bfs_source(R, C, N, s, dist, sigma)
    return dist, sigma


def brandes(R, C):
    N = len(R) - 1
    bc = np.empty(N, np.float64)
    lib().or_brandes(R, C, N, bc)
    return bc


# ------------------------------------------- subject-size restatements
_big = None


def big_lib():
    """liboracle_big.so (oracle_big.c): threaded, vectorised restatements with
    the results of the functions above, for subjects of tens of thousands of
    voxels."""
    global _big
    if _big is None:
        path = os.path.join(HERE, "liboracle_big.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "big"], check=True)
        L = _load(path)
        L.or_big_topk.argtypes = [_f64p, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int64, ct.c_int,
                                  _f64p, _i32p, _i32p]
        L.or_big_topk.restype = ct.c_int64
        L.or_brandes_mt.argtypes = [_i32p, _i32p, ct.c_int, ct.c_int, _f64p, _vp]
        _big = L
    return _big


def big_topk(z, kmax, abs_mode=False, weighted=False, threads=None):
    """The kmax pairs of largest key (r or |r|) in (key desc, i asc, j asc)
    order; the first k of them are graph_k's edge set for k edges and
    keys[k-1] its tau."""
    z = np.ascontiguousarray(z, np.float64)
    N, T = z.shape
    kmax = min(int(kmax), N * (N - 1) // 2)
    keys = np.empty(max(kmax, 1), np.float64)
    ii = np.empty(max(kmax, 1), np.int32)
    jj = np.empty(max(kmax, 1), np.int32)
    n = big_lib().or_big_topk(z, N, T, int(abs_mode), int(weighted), kmax, threads or os.cpu_count() or 1,
                              keys, ii, jj)
    if n < 0:
        raise MemoryError("or_big_topk ran out of memory")
    return keys[:n], ii[:n], jj[:n]


def csr_from_pairs(N, ii, jj):
    """Binary CSR (both directions, ascending columns) of undirected pairs."""
    u = np.concatenate([ii, jj]).astype(np.int64)
    v = np.concatenate([jj, ii]).astype(np.int64)
    order = np.argsort(u * N + v, kind="stable")
    C = v[order].astype(np.int32)
    R = np.zeros(N + 1, np.int64)
    np.add.at(R, u + 1, 1)
    return np.cumsum(R).astype(np.int32), C


def brandes_mt(R, C, threads=None, with_inv_sum=False):
    """or_brandes with the sources split over threads; with_inv_sum also
    returns sum_v 1/d(s, v) per source (or_bfs_paths' inv_sum)."""
    N = len(R) - 1
    bc = np.empty(N, np.float64)
    inv = np.empty(N, np.float64) if with_inv_sum else None
    big_lib().or_brandes_mt(np.ascontiguousarray(R, np.int32), np.ascontiguousarray(C, np.int32), N,
                            threads or os.cpu_count() or 1, bc, _ptr(inv))
    return (bc, inv) if with_inv_sum else bc


def fw_dense(d):
    d = np.ascontiguousarray(d, dtype=np.float32).copy()
    lib().or_fw_dense(d, d.shape[0])
    return d


def weighted_paths(R, C, V):
    N = len(R) - 1
    eff = np.empty(N, np.float32)
    lp = ct.c_double()
    if lib().or_weighted_paths(R, C, V, N, eff, ct.byref(lp)) != 0:
        raise MemoryError("dense distance matrix too large for the oracle")
    return eff, lp.value


def newman(R, C, gpu_rule_above=25000):
    N = len(R) - 1
    labels = np.empty(N, np.int32)
    Q = ct.c_double()
    nm = ct.c_int()
    nr = ct.c_int()
    lib().or_newman(R, C, N, gpu_rule_above, labels, ct.byref(Q), ct.byref(nm), ct.byref(nr))
    return labels, Q.value, nm.value, nr.value


def newman_weighted(R, C, Vw, gpu_rule_above=25000):
    """The weighted Newman tool's partition (or_newman_weighted); Vw is the
    value array the tool indexes by position."""
    R = np.ascontiguousarray(R, np.int32)
    C = np.ascontiguousarray(C, np.int32)
    Vw = np.ascontiguousarray(Vw, np.float32)
    N = len(R) - 1
    labels = np.zeros(max(N, 1), np.int32)
    Q, nm, nr = ct.c_double(), ct.c_int(), ct.c_int()
    lib().or_newman_weighted(R, C, Vw, len(Vw), N, gpu_rule_above, labels, ct.byref(Q), ct.byref(nm), ct.byref(nr))
    return labels[:N], Q.value, nm.value


def maslov(R, C, V, seed, attempts):
    N = len(R) - 1
    Ro = np.empty(N + 1, np.int32)
    Co = np.empty(max(len(C), 1), np.int32)
    Vo = np.empty(max(len(C), 1), np.float32) if V is not None else None
    ncommit = lib().or_maslov(R, C, _ptr(V), N, seed, attempts, Ro, Co, _ptr(Vo))
    return Ro, Co[: len(C)].copy(), (Vo[: len(C)].copy() if V is not None else None), ncommit


def rewire_seq(R, C, V, seed, attempts=None):
    """The reference's sequential Rewire with its 15-bit rand() stream seeded
    by `seed` (or_rewire_seq); attempts defaults to the reference's 2M."""
    N = len(R) - 1
    attempts = len(C) if attempts is None else attempts
    Ro = np.empty(N + 1, np.int32)
    Co = np.empty(max(len(C), 1), np.int32)
    Vo = np.empty(max(len(C), 1), np.float32) if V is not None else None
    ncommit = lib().or_rewire_seq(R, C, _ptr(V), N, seed, attempts, Ro, Co, _ptr(Vo))
    return Ro, Co[: len(C)].copy(), (Vo[: len(C)].copy() if V is not None else None), ncommit


def maslov_round_size(M):
    return int(lib().or_maslov_round_size(M))


def eigen_centrality(R, C, V=None, raw=False):
    """Power-method eigenvector centrality of the CUEC tools (or_eigen_centrality):
    returns (ec, eigenvalue, iterations, residual)."""
    R = np.ascontiguousarray(R, np.int32)
    C = np.ascontiguousarray(C, np.int32)
    N = len(R) - 1
    Vc = None if V is None else np.ascontiguousarray(V, np.float32)
    ec = np.zeros(max(N, 1), np.float64)
    lam, res = ct.c_double(0.0), ct.c_double(0.0)
    it = lib().or_eigen_centrality(R, C, _ptr(Vc), N, int(bool(raw)), ec, ct.byref(lam), ct.byref(res))
    return ec[:N], lam.value, int(it), res.value


# ------------------------------------------------------------ compiled reference
class _QuietFd:
    """Silences fd 1 around a reference call that prints."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


class Ref:
    """The reference's own CPU functions (oracle/_ref/)."""

    def __init__(self):
        self._cucormat = _load(os.path.join(REF_DIR, "libref_cucormat.so"))
        self._cormat_cpu = _load(os.path.join(REF_DIR, "libref_cormat_cpu.so"))
        self._metrics = _load(os.path.join(REF_DIR, "libref_metrics.so"))
        self._weighted = _load(os.path.join(REF_DIR, "libref_weighted.so"))
        self._wcormat = _load(os.path.join(REF_DIR, "libref_wcormat.so"))
        c = self._cucormat
        c.ref_cormat_cpu.argtypes = [_f32p, _f32p, ct.c_int, ct.c_int]
        c.ref_form_graph_r.argtypes = [_f32p, ct.c_int, ct.c_float, _i32p, _i32p, ct.c_longlong]
        c.ref_form_graph_r.restype = ct.c_longlong
        c.ref_form_graph_s.argtypes = [_f32p, ct.c_int, ct.c_longlong, _i32p, _i32p,
                                       ct.POINTER(ct.c_float), ct.c_longlong]
        c.ref_form_graph_s.restype = ct.c_longlong
        m = self._cormat_cpu
        m.ref_cormat_cpu_mt.argtypes = [_f32p, _f32p, ct.c_int, ct.c_int, ct.c_int]
        m.ref_form_graph_abs.argtypes = [_f32p, ct.c_int, ct.c_float, _i32p, _i32p, ct.c_longlong]
        m.ref_form_graph_abs.restype = ct.c_longlong
        g = self._metrics
        g.ref_betweenness.argtypes = [_i32p, _i32p, ct.c_int, ct.c_int, _f32p]
        g.ref_cp.argtypes = [_i32p, _i32p, ct.c_int, _f32p]
        g.ref_cp.restype = ct.c_double
        g.ref_apsp_bfs.argtypes = [_i32p, _i32p, ct.c_int, _f32p]
        g.ref_apsp_bfs.restype = ct.c_double
        g.ref_partition.argtypes = [_i32p, _i32p, ct.c_int, _i32p]
        w = self._weighted
        w.ref_cp2.argtypes = [_i32p, _i32p, _f32p, ct.c_int, _f32p]
        w.ref_cp2.restype = ct.c_double
        w.ref_bfw.argtypes = [_i32p, _i32p, _f32p, ct.c_int, ct.c_int, _f32p]
        x = self._wcormat
        x.ref_wform_graph_r.argtypes = [_f32p, ct.c_int, ct.c_float, _i32p, _i32p, _f32p, ct.c_longlong]
        x.ref_wform_graph_r.restype = ct.c_longlong
        for lib_, pre in ((c, "ref_"), (x, "ref_w")):
            getattr(lib_, pre + "cohort_add").argtypes = [_f32p, _f32p, ct.c_int, ct.c_int]
            getattr(lib_, pre + "cohort_finish").argtypes = [_f32p, ct.c_longlong, ct.c_int, ct.c_int]
        ms = os.path.join(REF_DIR, "libref_maslov.so")
        self._maslov = _load(ms) if os.path.exists(ms) else None
        if self._maslov is not None:
            self._maslov.ref_maslov.argtypes = [_i32p, _i32p, ct.c_int, ct.c_int, ct.c_uint, _i32p, _i32p]
        wms = os.path.join(REF_DIR, "libref_wmaslov.so")
        self._wmaslov = _load(wms) if os.path.exists(wms) else None
        if self._wmaslov is not None:
            self._wmaslov.ref_wmaslov.argtypes = [_i32p, _i32p, _f32p, ct.c_int, ct.c_int, ct.c_uint, _i32p, _i32p,
                                                  _f32p]
        wn = os.path.join(REF_DIR, "libref_wnewman.so")
        self._wnewman = _load(wn) if os.path.exists(wn) else None
        if self._wnewman is not None:
            self._wnewman.ref_wpartition.argtypes = [_i32p, _i32p, _f32p, ct.c_int, _i32p]

    @staticmethod
    def available() -> bool:
        return all(os.path.exists(os.path.join(REF_DIR, f"libref_{n}.so"))
                   for n in ("cucormat", "cormat_cpu", "metrics", "weighted", "wcormat"))

    def cormat_cpu(self, bold_TxN):
        bold = np.ascontiguousarray(bold_TxN, np.float32)
        T, N = bold.shape
        out = np.zeros(N * (N - 1) // 2, np.float32)
        self._cucormat.ref_cormat_cpu(out, bold, N, T)
        return out

    def cormat_cpu_mt(self, bold_TxN, threads):
        bold = np.ascontiguousarray(bold_TxN, np.float32)
        T, N = bold.shape
        out = np.zeros(N * (N - 1) // 2, np.float32)
        self._cormat_cpu.ref_cormat_cpu_mt(out, bold, N, T, threads)
        return out

    def graph_r(self, cormat, N, thr):
        cap = N * (N - 1)
        R = np.zeros(N + 1, np.int32)
        C = np.zeros(max(cap, 1), np.int32)
        nnz = self._cucormat.ref_form_graph_r(cormat, N, thr, R, C, cap)
        return R, C[:nnz].copy()

    def graph_abs(self, cormat, N, thr):
        cap = N * (N - 1)
        R = np.zeros(N + 1, np.int32)
        C = np.zeros(max(cap, 1), np.int32)
        nnz = self._cormat_cpu.ref_form_graph_abs(cormat, N, thr, R, C, cap)
        return R, C[:nnz].copy()

    def graph_s(self, cormat, N, k):
        cap = N * (N - 1)
        R = np.zeros(N + 1, np.int32)
        C = np.zeros(max(cap, 1), np.int32)
        tau = ct.c_float()
        nnz = self._cucormat.ref_form_graph_s(cormat, N, k, R, C, ct.byref(tau), cap)
        return R, C[:nnz].copy(), tau.value

    def wgraph_r(self, cormat, N, thr):
        cap = N * (N - 1)
        R = np.zeros(N + 1, np.int32)
        C = np.zeros(max(cap, 1), np.int32)
        V = np.zeros(max(cap, 1), np.float32)
        nnz = self._wcormat.ref_wform_graph_r(cormat, N, thr, R, C, V, cap)
        return R, C[:nnz].copy(), V[:nnz].copy()

    def betweenness(self, R, C):
        N = len(R) - 1
        bc = np.zeros(N, np.float32)
        self._metrics.ref_betweenness(R, C, N, int(R[-1]), bc)
        return bc

    def cp(self, R, C):
        N = len(R) - 1
        cp = np.zeros(N, np.float32)
        mean = self._metrics.ref_cp(R, C, N, cp)
        return cp, mean

    def apsp_bfs(self, R, C):
        N = len(R) - 1
        li = np.zeros(N, np.float32)
        lp = self._metrics.ref_apsp_bfs(R, C, N, li)
        return li, lp

    def partition(self, R, C):
        N = len(R) - 1
        res = np.zeros(N, np.int32)
        self._metrics.ref_partition(R, C, N, res)
        return res

    def wpartition(self, R, C, V):
        """The weighted tool's CPU Partition (every group on the CPU rule);
        None when libref_wnewman.so was not built."""
        if self._wnewman is None:
            return None
        N = len(R) - 1
        res = np.zeros(N, np.int32)
        self._wnewman.ref_wpartition(np.ascontiguousarray(R, np.int32), np.ascontiguousarray(C, np.int32),
                                     np.ascontiguousarray(V, np.float32), N, res)
        return res

    def cohort(self, r_subjects, N, fisher, weighted=False):
        """The reference's averaging branch (post_block with fisher_trans, then
        division and inv_fisher_trans) over float packed r of each subject."""
        M1 = N * (N - 1) // 2
        lib_, pre = (self._wcormat, "ref_w") if weighted else (self._cucormat, "ref_")
        cm = np.zeros(max(M1, 1), np.float32)
        for r in r_subjects:
            getattr(lib_, pre + "cohort_add")(cm, np.ascontiguousarray(r, np.float32), N, int(fisher))
        getattr(lib_, pre + "cohort_finish")(cm, M1, len(r_subjects), int(fisher))
        return cm[:M1]

    def maslov(self, R, C, seed, V=None):
        """The reference's Maslov (U) or Maslov_weighted_1 (W) with rand()
        seeded by `seed`: 2M attempts, (R, C[, V]) of the surrogate."""
        N = len(R) - 1
        R = np.ascontiguousarray(R, np.int32)
        C = np.ascontiguousarray(C, np.int32)
        Ro = np.empty(N + 1, np.int32)
        Co = np.empty(max(len(C), 1), np.int32)
        if V is None:
            self._maslov.ref_maslov(R, C, N, len(C), seed, Ro, Co)
            return Ro, Co[: len(C)].copy()
        Vo = np.empty(max(len(C), 1), np.float32)
        with _QuietFd():
            self._wmaslov.ref_wmaslov(R, C, np.ascontiguousarray(V, np.float32), N, len(C), seed, Ro, Co, Vo)
        return Ro, Co[: len(C)].copy(), Vo[: len(C)].copy()

    def cp2(self, R, C, V):
        N = len(R) - 1
        cp = np.zeros(N, np.float32)
        mean = self._weighted.ref_cp2(R, C, V, N, cp)
        return cp, mean

    def bfw(self, R, C, V, block=32):
        N = len(R) - 1
        d = np.zeros((N, N), np.float32)
        self._weighted.ref_bfw(R, C, V, N, block, d)
        return d


def participation(R, C, V, module):
    """PC_CPU's participation coefficient (or_participation): returns
    (pc, pc_normalised, n_modules), float32."""
    R = np.ascontiguousarray(R, np.int32)
    C = np.ascontiguousarray(C, np.int32)
    N = len(R) - 1
    Vc = None if V is None else np.ascontiguousarray(V, np.float32)
    mod = np.ascontiguousarray(module, np.float32)
    pc = np.zeros(max(N, 1), np.float32)
    pn = np.zeros(max(N, 1), np.float32)
    K = lib().or_participation(R, C, _ptr(Vc), N, mod, pc, pn)
    return pc[:N], pn[:N], int(K)


def fp64_fn(name, xs):
    """Elementwise or_ln / or_exp / or_fisher / or_inv_fisher over an array."""
    f = getattr(lib(), "or_" + name)
    return np.array([f(float(x)) for x in np.asarray(xs, np.float64).ravel()], np.float64)


def cohort_keys(bolds, fisher=False, weighted=False):
    """Subject-averaged keys of CUCorMat's to_average branch
    (or_cohort_add / or_cohort_finish): packed upper triangle, FP64.
    bolds: list of (T_s, N) float32 series with the same N."""
    N = bolds[0].shape[1]
    M1 = N * (N - 1) // 2
    acc = np.zeros(max(M1, 1), np.float64)
    for b in bolds:
        z, _ = zscore(b)
        lib().or_cohort_add(np.ascontiguousarray(z), N, z.shape[1], int(weighted), int(fisher), acc)
    key = np.zeros(max(M1, 1), np.float64)
    lib().or_cohort_finish(acc, M1, len(bolds), int(fisher), key)
    return key[:M1]
