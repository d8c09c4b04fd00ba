/*
 * oracle.c -- CPU restatement of the PAGANI hot path (FP64 where the text says
 * so).  TEST INFRASTRUCTURE ONLY: this is the checker used by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline/reference legs.  The
 * product library never links it.
 *
 * Every function names the reference function it restates.  Paths are relative
 * to the reference project root:
 *   U/ = src/BNAPlatform-win64-cuda7.0-20151118/src/
 *   W/ = src/BNAPlatform-weighted-network-win64-cuda7.0-20151118/src/
 *
 * Pinning: tests/test_oracle_ref.py compares these functions with the
 * reference's own CPU sources compiled by oracle/Makefile into oracle/_ref/,
 * and tests/golden/ holds fixtures generated from that compiled reference.
 *
 * Build: gcc -O2 -ffp-contract=off: no multiply-add is fused except where
 * fma() is written out (the r accumulation).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <limits.h>

/* ---------------------------------------------------------------- z-score */
/* Restates the normalisation loop of CorMat_gpu, U/CorMat/CUCorMat/CUCORMAT/
 * CorMat.cu:34-53 (same as CorMat_cpu, CorMat.cpp:872-890): FP64 mean and
 * root of the sum of squares, z = (x - mean) / s.  The reference stores z as
 * float; the oracle keeps it in FP64.  A row with s == 0 (or NaN input) gives
 * NaN r in the reference, which post_block (CorMat.cpp:821) then stores as 0;
 * here the row becomes the zero vector so that every r involving it is 0. */
int or_zscore(const float* bold, int N, int T, double* z)
{
    int zero = 0;
    for (int i = 0; i < N; i++) {
        double s1 = 0.0, s2 = 0.0;
        for (int t = 0; t < T; t++) s1 += (double)bold[(int64_t)t * N + i];
        s1 /= T;
        for (int t = 0; t < T; t++) {
            double d = (double)bold[(int64_t)t * N + i] - s1;
            s2 += d * d;
        }
        s2 = sqrt(s2);
        double* zi = z + (int64_t)i * T;
        if (!(s2 > 0.0) || !isfinite(s2)) {
            zero++;
            for (int t = 0; t < T; t++) zi[t] = 0.0;
            continue;
        }
        for (int t = 0; t < T; t++) zi[t] = ((double)bold[(int64_t)t * N + i] - s1) / s2;
    }
    return zero;
}

/* Range rule of post_block: unweighted keeps r in [-1, 1]
 * (U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:821-822); weighted keeps r in
 * (-1-1e-6, 1+1e-6) (W/CorMat/CUCorMat/CUCorMat/CorMat.cpp:821-822 with
 * ep = 1e-6 from :17).  Anything else (including NaN) is stored as 0. */
static inline double range_rule(double r, int weighted)
{
    if (weighted) return (r > -1.0 - 1e-6 && r < 1.0 + 1e-6) ? r : 0.0;
    return (r >= -1.0 && r <= 1.0) ? r : 0.0;
}

double or_pair_r(const double* z, int T, int i, int j, int weighted)
{
    const double* a = z + (int64_t)i * T;
    const double* b = z + (int64_t)j * T;
    double r = 0.0;
    for (int t = 0; t < T; t++) r = fma(a[t], b[t], r);
    return range_rule(r, weighted);
}

/* Packed upper triangle, row-major, i < j: the .cormat layout
 * (CorMat.cpp:285-294, manual p11). */
void or_corr_packed(const double* z, int N, int T, int weighted, double* r)
{
    int64_t k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) r[k++] = or_pair_r(z, T, i, j, weighted);
}

/* Edge count for a sparsity threshold, exactly as main() computes it,
 * CorMat.cpp:310-312: Clength = (long long)2*M1*s/100.0 -- the long long
 * product is converted to float and multiplied by the float s in single
 * precision before the double division -- then rounded up to even.  The
 * number of undirected edges is Clength/2. */
int64_t or_sparsity_k(int N, float s)
{
    long long M1 = (long long)(N - 1) * N / 2;
    float prod = (float)(2LL * M1) * s;
    long long Clength = (long long)((double)prod / 100.0);
    Clength += Clength % 2;
    return Clength / 2;
}

/* Weighted r threshold: W/CorMat/CUCorMat/CUCorMat/CorMat.cpp:310 passes
 * r_thresh - ep (double) to a float parameter, so the effective threshold is
 * the float nearest to thr - 1e-6. */
float or_weighted_r_threshold(float thr) { return (float)((double)thr - 1e-6); }

static inline double keyof(double r, int abs_mode) { return abs_mode ? fabs(r) : r; }

/* Append undirected edge (i, j), i < j, in lexicographic pair order; rows end
 * up with ascending columns, matching FormCSRGraph's O(N^2) scan
 * (CorMat.cpp:839-857; weighted V from the packed r, W CorMat.cpp:853-882). */
static int64_t build_csr(const double* r, int N, const unsigned char* keep, int abs_mode,
                         int32_t* R, int32_t* C, float* V, int64_t cap)
{
    int64_t M1 = (int64_t)N * (N - 1) / 2;
    int64_t* deg = (int64_t*)calloc((size_t)N + 1, sizeof(int64_t));
    int64_t k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++, k++)
            if (keep[k]) { deg[i]++; deg[j]++; }
    int64_t nnz = 0;
    for (int i = 0; i < N; i++) nnz += deg[i];
    if (nnz > cap || nnz > INT32_MAX) { free(deg); return -1; }
    R[0] = 0;
    for (int i = 0; i < N; i++) R[i + 1] = R[i] + (int32_t)deg[i];
    int64_t* cur = deg;
    for (int i = 0; i < N; i++) cur[i] = R[i];
    k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++, k++)
            if (keep[k]) {
                float w = (float)(abs_mode ? fabs(r[k]) : r[k]);
                C[cur[i]] = j; if (V) V[cur[i]] = w; cur[i]++;
                C[cur[j]] = i; if (V) V[cur[j]] = w; cur[j]++;
            }
    (void)M1;
    free(deg);
    return nnz;
}

/* r-threshold graph: FormFullGraph, CorMat.cpp:633-653 (strict r > thr).
 * abs_mode thresholds |r| instead, as CorMat_CPU does
 * (U/CorMat/CorMat_CPU/CorMat/CorMat_CPU.cpp:198). */
int64_t or_graph_r(const double* r, int N, double thr, int abs_mode,
                   int32_t* R, int32_t* C, float* V, int64_t cap)
{
    int64_t M1 = (int64_t)N * (N - 1) / 2;
    unsigned char* keep = (unsigned char*)malloc((size_t)(M1 > 0 ? M1 : 1));
    for (int64_t k = 0; k < M1; k++) keep[k] = keyof(r[k], abs_mode) > thr;
    int64_t nnz = build_csr(r, N, keep, abs_mode, R, C, V, cap);
    free(keep);
    return nnz;
}

static int cmp_desc(const void* a, const void* b)
{
    double x = *(const double*)a, y = *(const double*)b;
    return (x < y) - (x > y);
}

/* Sparsity graph: select + FormFullGraph_s, CorMat.cpp:655-773.  tau is the
 * k-th largest key; every pair with key > tau is kept, and of the pairs with
 * key == tau only the lexicographically first (k - #above) survive -- the
 * reference pops the most recently pushed tie whenever the count exceeds k
 * (:748-759), which leaves exactly the earliest ties. */
int64_t or_graph_k(const double* r, int N, int64_t k, int abs_mode, double* tau,
                   int32_t* R, int32_t* C, float* V, int64_t cap)
{
    int64_t M1 = (int64_t)N * (N - 1) / 2;
    unsigned char* keep = (unsigned char*)calloc((size_t)(M1 > 0 ? M1 : 1), 1);
    double t = INFINITY;
    if (k > 0 && M1 > 0) {
        if (k > M1) k = M1;
        double* s = (double*)malloc((size_t)M1 * sizeof(double));
        for (int64_t q = 0; q < M1; q++) s[q] = keyof(r[q], abs_mode);
        qsort(s, (size_t)M1, sizeof(double), cmp_desc);
        t = s[k - 1];
        int64_t above = 0;
        for (int64_t q = 0; q < M1; q++) above += s[q] > t;
        free(s);
        int64_t ties = k - above;
        for (int64_t q = 0; q < M1; q++) {
            double x = keyof(r[q], abs_mode);
            if (x > t) keep[q] = 1;
            else if (x == t && ties > 0) { keep[q] = 1; ties--; }
        }
    }
    if (tau) *tau = t;
    int64_t nnz = build_csr(r, N, keep, abs_mode, R, C, V, cap);
    free(keep);
    return nnz;
}

/* ------------------------------------------------- cohort (subject average) */
/* FP64 natural logarithm and exponential from +, -, *, / alone, so that this
 * restatement and the device code round identically.  The method is the
 * classical argument reduction (Cody & Waite, "Software Manual for the
 * Elementary Functions", 1980):
 *   ln x  = e ln2 + 2 atanh(s),  x = m 2^e,  m in [sqrt(1/2), sqrt(2)),
 *           s = (m - 1) / (m + 1), atanh by its odd Taylor series to s^23
 *           (|s| <= 0.1716: truncation below 2^-60 relative);
 *   exp x = 2^k e^t,  k = x / ln2 rounded half away from zero,
 *           t = (x - k ln2_hi) - k ln2_lo, e^t by its Taylor series to t^14
 *           (|t| <= 0.347).
 * ln2_hi keeps 42 significant bits, so k ln2_hi is exact for |k| < 2^11.
 * The coefficients are 2/(2j+1) and 1/n!, rounded to nearest.  Measured
 * against the C library: ln within 2 ulp, exp within 1 ulp. */
static const double LN2_HI = 0x1.62e42fefa3800p-1, LN2_LO = 0x1.ef35793c76730p-45;
static const double INV_LN2 = 0x1.71547652b82fep+0, SQRT2 = 0x1.6a09e667f3bcdp+0;
static const double ATANH_C[11] = {   /* 2/3, 2/5, ..., 2/23 */
    0x1.5555555555555p-1, 0x1.999999999999ap-2, 0x1.2492492492492p-2, 0x1.c71c71c71c71cp-3,
    0x1.745d1745d1746p-3, 0x1.3b13b13b13b14p-3, 0x1.1111111111111p-3, 0x1.e1e1e1e1e1e1ep-4,
    0x1.af286bca1af28p-4, 0x1.8618618618618p-4, 0x1.642c8590b2164p-4};
static const double EXP_C[15] = {     /* 1/n!, n = 0..14 */
    0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p-1, 0x1.5555555555555p-3,
    0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
    0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
    0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37};

static double pow2i(int k)   /* 2^k for -1022 <= k <= 1023 */
{
    uint64_t u = (uint64_t)(k + 1023) << 52;
    double d;
    memcpy(&d, &u, 8);
    return d;
}

double or_ln(double x)
{
    if (x != x || x < 0.0) return NAN;
    if (x == 0.0) return -INFINITY;
    if (isinf(x)) return x;
    uint64_t u;
    memcpy(&u, &x, 8);
    int e = 0;
    if (((u >> 52) & 0x7ff) == 0) {  /* subnormal: scale by 2^54 first */
        x = x * 0x1p54;
        memcpy(&u, &x, 8);
        e = -54;
    }
    e += (int)((u >> 52) & 0x7ff) - 1023;
    u = (u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &u, 8);
    if (m > SQRT2) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    double p = ATANH_C[10];
    for (int j = 9; j >= 0; j--) p = ATANH_C[j] + s2 * p;
    double ls = 2.0 * s + s * (s2 * p);
    double de = (double)e;
    return de * LN2_HI + (de * LN2_LO + ls);
}

double or_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.2) return 0.0;
    double kd = x * INV_LN2;
    long long k = (long long)(kd + (kd >= 0.0 ? 0.5 : -0.5));
    double dk = (double)k;
    double t = (x - dk * LN2_HI) - dk * LN2_LO;
    double p = EXP_C[14];
    for (int n = 13; n >= 0; n--) p = EXP_C[n] + t * p;
    if (k > 1023) return p * pow2i(1023) * pow2i((int)k - 1023);
    if (k < -1022) return p * pow2i((int)k + 600) * pow2i(-600);
    return p * pow2i((int)k);
}

/* fisher_trans, U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:35-41 (W :35-41 as
 * fishertrans), in FP64: r == 1 becomes 1 - 1e-6, z = 0.5 ln((1+r)/(1-r)).
 * Under the weighted range rule r may lie in (1, 1+1e-6) or (-1-1e-6, -1],
 * where the reference's float log returns NaN; here r >= 1 is treated like
 * r == 1 and r <= -1 gives -inf (what r == -1 gives in the reference). */
double or_fisher(double r)
{
    if (r >= 1.0) r = 1.0 - 1e-6;
    if (r <= -1.0) return -INFINITY;
    return 0.5 * or_ln((1.0 + r) / (1.0 - r));
}

/* inv_fisher_trans, CorMat.cpp:43-49: r = (e^{2z} - 1) / (e^{2z} + 1). */
double or_inv_fisher(double z)
{
    double e = or_exp(2.0 * z);
    return (e - 1.0) / (e + 1.0);
}

/* One subject of the averaging branch of CUCorMat's main()
 * (U CorMat.cpp:380-470, W :386-476): post_block (:775-838) adds, for every
 * pair, r (to_average yn/bn) or fisher_trans(r) (yf/bf) to the running sum
 * when r passes the range rule (an r that fails it adds nothing, which equals
 * adding the 0 of range_rule: fisher(0) = 0).  Here the sum is FP64 and the
 * subjects are added in call order. */
void or_cohort_add(const double* z, int N, int T, int weighted, int fisher, double* acc)
{
    int64_t k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++, k++) {
            double r = or_pair_r(z, T, i, j, weighted);
            acc[k] += fisher ? or_fisher(r) : r;
        }
}

/* The end of the averaging branch (U CorMat.cpp:514-524, W :514-524): the
 * sum divided by the subject count, then inv_fisher_trans for yf/bf.  The
 * result is the key that FormFullGraph / FormFullGraph_s threshold (signed)
 * and, in the weighted tool, the edge value. */
void or_cohort_finish(const double* acc, int64_t M1, int subjects, int fisher, double* key)
{
    for (int64_t k = 0; k < M1; k++) {
        double a = acc[k] / (double)subjects;
        key[k] = fisher ? or_inv_fisher(a) : a;
    }
}

/* ----------------------------------------------------------------- degree */
/* U/Degree/Degree/Degree.cpp:85-91: (float)R[k+1] - R[k]; isolated count.
 * W/Degree/Degree/Degree.cpp:82-88: strength = float sum of V in CSR order. */
void or_degree(const int32_t* R, const float* V, int N, float* deg, int32_t* isolated)
{
    int32_t iso = 0;
    for (int k = 0; k < N; k++) {
        if (V) {
            float s = 0.0f;
            for (int32_t e = R[k]; e < R[k + 1]; e++) s += V[e];
            deg[k] = s;
        } else {
            deg[k] = (float)R[k + 1] - (float)R[k];
        }
        if (R[k + 1] == R[k]) iso++;
    }
    if (isolated) *isolated = iso;
}

/* ------------------------------------------------------- binary clustering */
/* U/Cp/Cp/Cp.cpp:78-116: t_k = number of connected neighbour pairs,
 * Cp[k] = (double)t / k / (k-1) * 2 stored as float, 0 when k < 2; mean over
 * all N nodes (:64-72).  The mean here is the sequential FP64 sum of the
 * float Cp values. */
void or_cp_binary(const int32_t* R, const int32_t* C, int N, int64_t* tri, float* cp, double* mean)
{
    int32_t* mark = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    for (int i = 0; i < N; i++) mark[i] = -1;
    double sum = 0.0;
    for (int u = 0; u < N; u++) {
        int32_t k = R[u + 1] - R[u];
        for (int32_t e = R[u]; e < R[u + 1]; e++) mark[C[e]] = u;
        int64_t twice = 0;
        for (int32_t e = R[u]; e < R[u + 1]; e++) {
            int32_t v = C[e];
            for (int32_t f = R[v]; f < R[v + 1]; f++) twice += (mark[C[f]] == u);
        }
        int64_t t = twice / 2;
        if (tri) tri[u] = t;
        float c = 0.0f;
        if (k >= 2) {
            double x = (double)t;
            x = x / k;
            x = x / (k - 1);
            x = x * 2;
            c = (float)x;
        }
        cp[u] = c;
        sum += (double)c;
    }
    free(mark);
    if (mean) *mean = N > 0 ? sum / N : 0.0;
}

/* ------------------------------------------------------- Onnela clustering */
/* W/Cp/Cp/Cp_2.cpp:23-130: w_hat = V / V_max (float division), per node the
 * sum over connected neighbour pairs j < h of (w_hat_jh w_hat_kj w_hat_kh)^(1/3)
 * (:123), Cp = 2 sum / k / (k-1) (:125).  vmax_first_n = 1 reproduces the
 * reference CPU's maximum over V[0..N) only (:27-30); 0 takes the maximum over
 * all edges as the GPU tool does (W/Cp_GPU/CUCP/Cp.cu cublasIsamax).  The
 * per-node sum is FP64 here (the reference accumulates in float). */
void or_onnela(const int32_t* R, const int32_t* C, const float* V, int N, int vmax_first_n,
               float* cp, double* mean)
{
    int64_t nnz = R[N];
    float vmax = 0.0f;
    int64_t lim = vmax_first_n ? (N < nnz ? N : nnz) : nnz;
    if (lim > 0) {
        vmax = V[0];
        for (int64_t e = 1; e < lim; e++) if (vmax < V[e]) vmax = V[e];
    }
    float* wh = (float*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(float));
    for (int64_t e = 0; e < nnz; e++) wh[e] = V[e] / vmax;
    float* roww = (float*)calloc((size_t)N, sizeof(float));
    int32_t* mark = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    for (int i = 0; i < N; i++) mark[i] = -1;
    double sum = 0.0;
    for (int u = 0; u < N; u++) {
        int32_t k = R[u + 1] - R[u];
        for (int32_t e = R[u]; e < R[u + 1]; e++) { mark[C[e]] = u; roww[C[e]] = wh[e]; }
        double acc = 0.0;
        for (int32_t e = R[u]; e < R[u + 1]; e++) {
            int32_t j = C[e];
            for (int32_t f = R[j]; f < R[j + 1]; f++) {
                int32_t h = C[f];
                if (h > j && mark[h] == u && wh[f] != 0.0f)
                    acc += pow((double)wh[f] * roww[j] * roww[h], 1.0 / 3);
            }
        }
        float c = 0.0f;
        if (k >= 2) c = (float)(2.0 * acc / k / (k - 1));
        cp[u] = c;
        sum += (double)c;
    }
    free(wh); free(roww); free(mark);
    if (mean) *mean = N > 0 ? sum / N : 0.0;
}

/* ------------------------------------------------- BFS path length (hops) */
/* U/BFS_MulCPU/BFS_MulCPU/APSP_BFS.cpp:27-192.  For every source a queue BFS
 * gives hop counts; unreachable pairs contribute nothing.  inv_sum[s] =
 * sum_v 1/d(s,v) (accumulated as sum_d count_d / d, d ascending);
 * Li = inv_sum / (N-1) (:126); Lp = N(N-1) / sum_s inv_sum[s], which equals
 * the reference's 1/(sum_{i<j} 1/d / N / (N-1)) / 2 (:135-138).
 * hop_hist[d] counts ordered pairs at distance d (d <= max_hop).
 * Returns the largest finite distance seen. */
int or_bfs_paths(const int32_t* R, const int32_t* C, int N, double* inv_sum,
                 int64_t* hop_hist, int max_hop, double* lp)
{
    int32_t* dist = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    int32_t* q = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    int64_t* cnt = (int64_t*)calloc((size_t)N + 1, sizeof(int64_t));
    int maxd = 0;
    double total = 0.0;
    if (hop_hist) memset(hop_hist, 0, sizeof(int64_t) * (size_t)(max_hop + 1));
    for (int s = 0; s < N; s++) {
        for (int i = 0; i < N; i++) dist[i] = -1;
        int head = 0, tail = 0, dmax = 0;
        dist[s] = 0; q[tail++] = s;
        while (head < tail) {
            int v = q[head++];
            for (int32_t e = R[v]; e < R[v + 1]; e++) {
                int w = C[e];
                if (dist[w] < 0) { dist[w] = dist[v] + 1; q[tail++] = w; cnt[dist[w]]++;
                                   if (dist[w] > dmax) dmax = dist[w]; }
            }
        }
        double acc = 0.0;
        for (int d = 1; d <= dmax; d++) {
            acc += (double)cnt[d] / d;
            if (hop_hist && d <= max_hop) hop_hist[d] += cnt[d];
            cnt[d] = 0;
        }
        if (dmax > maxd) maxd = dmax;
        if (inv_sum) inv_sum[s] = acc;
        total += acc;
    }
    if (lp) *lp = total > 0.0 ? (double)N * (N - 1) / total : 0.0;
    free(dist); free(q); free(cnt);
    return maxd;
}

/* Single-source hop distances and exact shortest-path counts (the forward
 * half of Betweenness_CPU, U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:37-56, with the
 * float sigma replaced by a 64-bit integer). */
int or_bfs_source(const int32_t* R, const int32_t* C, int N, int s, int32_t* dist, int64_t* sigma)
{
    int32_t* q = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    for (int i = 0; i < N; i++) { dist[i] = -1; sigma[i] = 0; }
    int head = 0, tail = 0, dmax = 0;
    dist[s] = 0; sigma[s] = 1; q[tail++] = s;
    while (head < tail) {
        int v = q[head++];
        for (int32_t e = R[v]; e < R[v + 1]; e++) {
            int w = C[e];
            if (dist[w] < 0) { dist[w] = dist[v] + 1; q[tail++] = w; if (dist[w] > dmax) dmax = dist[w]; }
            if (dist[w] == dist[v] + 1) sigma[w] += sigma[v];
        }
    }
    free(q);
    return dmax;
}

/* ------------------------------------------------------------- betweenness */
/* Brandes, U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:6-82: every vertex is a source and
 * BC[w] += delta[w] for w != s, i.e. the sum over ORDERED pairs (twice the
 * undirected textbook value).  sigma is exact int64 and delta FP64 (the
 * reference uses float for both). */
void or_brandes(const int32_t* R, const int32_t* C, int N, double* bc)
{
    int32_t* dist = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    int64_t* sigma = (int64_t*)malloc((size_t)N * sizeof(int64_t));
    double* delta = (double*)malloc((size_t)N * sizeof(double));
    int32_t* order = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    for (int i = 0; i < N; i++) bc[i] = 0.0;
    for (int s = 0; s < N; s++) {
        for (int i = 0; i < N; i++) { dist[i] = -1; sigma[i] = 0; delta[i] = 0.0; }
        int head = 0, tail = 0;
        dist[s] = 0; sigma[s] = 1; order[tail++] = s;
        while (head < tail) {
            int v = order[head++];
            for (int32_t e = R[v]; e < R[v + 1]; e++) {
                int w = C[e];
                if (dist[w] < 0) { dist[w] = dist[v] + 1; order[tail++] = w; }
                if (dist[w] == dist[v] + 1) sigma[w] += sigma[v];
            }
        }
        for (int p = tail - 1; p >= 0; p--) {
            int w = order[p];
            double acc = 0.0;
            for (int32_t e = R[w]; e < R[w + 1]; e++) {
                int v = C[e];
                if (dist[v] == dist[w] + 1) acc += (1.0 + delta[v]) / (double)sigma[v];
            }
            delta[w] = (double)sigma[w] * acc;
            if (w != s) bc[w] += delta[w];
        }
    }
    free(dist); free(sigma); free(delta); free(order);
}

/* ------------------------------------------------------- Floyd-Warshall */
/* Min-plus closure in FP32, BFW_one_block_C, W/Lp/CUBFW_Lp/CUBFW_Lp/BFW.cpp:26-39,
 * applied to one block covering the whole matrix (classic k-outer order). */
void or_fw_dense(float* d, int n)
{
    for (int k = 0; k < n; k++) {
        const float* dk = d + (int64_t)k * n;
        for (int i = 0; i < n; i++) {
            float* di = d + (int64_t)i * n;
            float dik = di[k];
            for (int j = 0; j < n; j++) {
                float c = dik + dk[j];
                if (c < di[j]) di[j] = c;
            }
        }
    }
}

/* Weighted path length: CUBFW_Lp, W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp.cpp:13-162.
 * Distance of an edge is 1/w (float, init_block FormBlock.cpp:64), 0 on the
 * diagonal, infinity elsewhere; APSP by min-plus; distances below 0.1 are
 * skipped (:77); eff[u] = sum_v 1/d(u,v) / (N-1), set to 0 when below 1/N
 * (:99-104); Lp = N(N-1) / sum_{u != v} 1/d (:107-109).  Sums are FP64. */
int or_weighted_paths(const int32_t* R, const int32_t* C, const float* V, int N,
                      float* eff, double* lp)
{
    float* d = (float*)malloc((size_t)N * N * sizeof(float));
    if (!d) return -1;
    for (int64_t q = 0; q < (int64_t)N * N; q++) d[q] = INFINITY;
    for (int i = 0; i < N; i++)
        for (int32_t e = R[i]; e < R[i + 1]; e++) d[(int64_t)i * N + C[e]] = 1.0f / V[e];
    for (int i = 0; i < N; i++) d[(int64_t)i * N + i] = 0.0f;
    or_fw_dense(d, N);
    double total = 0.0;
    for (int u = 0; u < N; u++) {
        double acc = 0.0;
        for (int v = 0; v < N; v++) {
            if (u == v) continue;
            float x = d[(int64_t)u * N + v];
            if (x < 0.1f) continue;
            acc += 1.0 / (double)x;
        }
        total += acc;
        float e = (float)(acc / (N - 1));
        if (e < 1.0f / N) e = 0.0f;
        if (eff) eff[u] = e;
    }
    if (lp) *lp = total > 0.0 ? 1.0 / (total / N / (N - 1)) : INFINITY;
    free(d);
    return 0;
}

/* ------------------------------------------------------ Newman modularity */
/* Leading-eigenvector bisection, restating Partition / Sub_Partition /
 * Lead_Vector of U/cuda_EC/cuda_EC/Modularity_CPU.cpp:48-298 with the
 * constants of :18-25 (MAX_ITER 10000, Epsilon 1e-6, LAMBDA 0.01,
 * MIN_GROUP 1) and the start vector v[i] = original node id (RANDOM_V0, :242).
 * The tool (modularity_GPU.cu:488) sends sub-graphs with more than 25,000
 * nodes to Sub_Partition_GPU, whose only rule change is the shift condition
 * lambda < -LAMBDA instead of lambda < 0 (modularity_GPU.cu:374 vs
 * Modularity_CPU.cpp:177); gpu_rule_above selects that threshold.
 * Q (:116-124) is computed from module degree sums: identical in exact
 * arithmetic to the reference's O(N^2) double loop. */
typedef struct {
    int N, M;
    const int32_t* R;
    double *v, *v0, *vv, *sumBG;
    int last_iter;
    double last_res;
    /* weighted tool (W/Newman_Modularity_GPU/CUmodularity): weights by
     * position in the full graph's value array, indexed by the sub-graph's
     * edge (groups above the GPU rule, modularity_GPU.cu:135) or by its row
     * (the CPU Lead_Vector, Modularity_CPU.cpp:261); positions past the array
     * count 0 */
    const float* Vw;
    int64_t wn;
    int wmode;   /* 0 none, 1 by row, 2 by edge */
} nm_state;

static double nm_norm(const double* x, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += x[i] * x[i];
    return sqrt(s);
}

static double nm_lead_vector(nm_state* st, const int32_t* sR, const int32_t* sC, int n,
                             const int32_t* AD, double beta)
{
    const int32_t* R = st->R;
    double *v = st->v, *v0 = st->v0, *vv = st->vv, *sumBG = st->sumBG;
    int M = st->M;
    for (int i = 0; i < n; i++) v[i] = AD[i];
    double err1 = 1, err2 = 1, vNorm = 0;
    int iter = 0;
    double* verr = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    while (err1 > 1e-6 && err2 > 1e-6 && iter < 10000) {
        for (int i = 0; i < n; i++) { v0[i] = v[i]; vv[AD[i]] = v[i]; }
        double v_k = 0;
        for (int i = 0; i < n; i++) v_k += v0[i] * (R[AD[i] + 1] - R[AD[i]]);
        for (int i = 0; i < n; i++) {
            double t = 0;
            if (st->wmode == 0) {
                for (int32_t j = sR[i]; j < sR[i + 1]; j++) t += vv[sC[j]];
            } else if (st->wmode == 2) {
                for (int32_t j = sR[i]; j < sR[i + 1]; j++) t += vv[sC[j]] * (j < st->wn ? (double)st->Vw[j] : 0.0);
            } else {
                const double w = i < st->wn ? (double)st->Vw[i] : 0.0;
                for (int32_t j = sR[i]; j < sR[i + 1]; j++) t += vv[sC[j]] * w;
            }
            t -= v_k / 2 / M * (R[AD[i] + 1] - R[AD[i]]) + (sumBG[i] - beta) * v0[i];
            v[i] = t;
        }
        vNorm = nm_norm(v, n);
        for (int i = 0; i < n; i++) v[i] = v[i] / vNorm;
        for (int i = 0; i < n; i++) verr[i] = v[i] - v0[i];
        err1 = nm_norm(verr, n);
        for (int i = 0; i < n; i++) verr[i] = v[i] + v0[i];
        err2 = nm_norm(verr, n);
        iter++;
    }
    free(verr);
    st->last_iter = iter;
    st->last_res = err1 < err2 ? err1 : err2;
    int mx = 0;
    for (int i = 0; i < n; i++) if (fabs(v[i]) > fabs(v[mx])) mx = i;
    return (v[mx] * v0[mx] > 0) ? vNorm : -vNorm;
}

static int newman_core(const int32_t* R, const int32_t* C, const float* Vw, int64_t wn, int N, int gpu_rule_above,
                       int32_t* labels, double* Qout, int* n_modules, int* n_rounds)
{
    int M = R[N] / 2;
    nm_state st;
    st.N = N; st.M = M; st.R = R;
    st.Vw = Vw; st.wn = wn; st.wmode = 0;
    st.v = (double*)calloc((size_t)N + 1, sizeof(double));
    st.v0 = (double*)calloc((size_t)N + 1, sizeof(double));
    st.vv = (double*)calloc((size_t)N + 1, sizeof(double));
    st.sumBG = (double*)calloc((size_t)N + 1, sizeof(double));
    int32_t* Result = labels;
    int32_t* Adjust = (int32_t*)calloc((size_t)N + 2, sizeof(int32_t));
    int32_t* AD = (int32_t*)malloc((size_t)(N + 1) * sizeof(int32_t));
    int32_t* sR = (int32_t*)malloc((size_t)(N + 1) * sizeof(int32_t));
    int32_t* sC = (int32_t*)malloc((size_t)(R[N] > 0 ? R[N] : 1) * sizeof(int32_t));
    unsigned char* G = (unsigned char*)malloc((size_t)(N > 0 ? N : 1));
    memset(Result, 0, sizeof(int32_t) * (size_t)N);
    int Round = 0, Max_Result = 0, Module_Num = 1, Index = 1;
    while (Round <= Max_Result) {
        long long innerM = 2LL * M;
        int NumG = 0;
        for (int i = 0; i < N; i++) {
            G[i] = (Result[i] == Round);
            if (G[i]) { AD[NumG++] = i; continue; }
            innerM -= R[i + 1] - R[i];
        }
        int nc = 0, nr = 0;
        sR[nr++] = 0;
        for (int i = 0; i < N; i++) {
            if (!G[i]) continue;
            for (int32_t j = R[i]; j < R[i + 1]; j++) if (G[C[j]]) sC[nc++] = C[j];
            sR[nr++] = nc;
        }
        if (NumG) {
            int n = NumG;
            for (int i = 0; i < n; i++)
                st.sumBG[i] = (sR[i + 1] - sR[i]) - (R[AD[i] + 1] - R[AD[i]]) * (double)innerM / 2 / M;
            st.wmode = Vw ? (n > gpu_rule_above ? 2 : 1) : 0;
            double lambda = nm_lead_vector(&st, sR, sC, n, AD, 0.0);
            double shift_below = (n > gpu_rule_above) ? -0.01 : 0.0;
            if (lambda < shift_below) lambda += nm_lead_vector(&st, sR, sC, n, AD, -lambda);
            long long subP = 0, subN = 0;
            for (int i = 0; i < n; i++) { subP += st.v[i] > 0; subN += st.v[i] <= 0; }
            int Issub = (lambda > 0.01 && subP > 1 && subN > 1);
            if (Issub) {
                for (int i = 0; i < n; i++)
                    Result[AD[i]] = Max_Result + 1 + (st.v[i] * (subP - subN + 0.5) <= 0);
                Max_Result += 2;
            } else {
                Adjust[Round] = Index++;
            }
            Module_Num += Issub;
        }
        Round++;
    }
    /* Q from module degree sums (before relabelling). */
    double Q = 0.0;
    if (M > 0) {
        int64_t inside = 0;
        double* Kc = (double*)calloc((size_t)Max_Result + 2, sizeof(double));
        for (int i = 0; i < N; i++) {
            for (int32_t j = R[i]; j < R[i + 1]; j++) inside += Result[i] == Result[C[j]];
            Kc[Result[i]] += R[i + 1] - R[i];
        }
        double sq = 0.0;
        for (int c = 0; c <= Max_Result; c++) sq += Kc[c] * Kc[c];
        Q = ((double)inside - sq / 2 / M) / (2.0 * M);
        free(Kc);
    }
    for (int i = 0; i < N; i++) Result[i] = Adjust[Result[i]];
    if (Qout) *Qout = Q;
    if (n_modules) *n_modules = Module_Num;
    if (n_rounds) *n_rounds = Round;
    free(st.v); free(st.v0); free(st.vv); free(st.sumBG);
    free(Adjust); free(AD); free(sR); free(sC); free(G);
    return 0;
}

int or_newman(const int32_t* R, const int32_t* C, int N, int gpu_rule_above,
              int32_t* labels, double* Qout, int* n_modules, int* n_rounds)
{
    return newman_core(R, C, NULL, 0, N, gpu_rule_above, labels, Qout, n_modules, n_rounds);
}

/* The weighted Newman tool: the same partition with the weights Vw[0..wn) in
 * the power iteration's products only (degrees, M and Q stay binary, as in
 * the reference). */
int or_newman_weighted(const int32_t* R, const int32_t* C, const float* Vw, int64_t wn, int N, int gpu_rule_above,
                       int32_t* labels, double* Qout, int* n_modules, int* n_rounds)
{
    return newman_core(R, C, Vw, wn, N, gpu_rule_above, labels, Qout, n_modules, n_rounds);
}

/* --------------------------------------------------------- Maslov rewiring */
/* Maslov-Sneppen rewiring: Rewire/Maslov,
 * U/cuda_EC/cuda_EC/Maslov.cpp:8-109 and the weighted variant
 * Maslov_weighted_1, W/Maslov/Maslov/Maslov.cpp:50-196 (weights stay with the
 * edge slot that carries them).  The reference draws from srand(time(0)) /
 * rand() and evaluates its attempts one after another.  This restatement
 * uses a seeded counter-based generator (attempt a: stream bits 2a and
 * 2a + 1) and the round schedule of the GPU kernel: a round
 * holds the attempts deferred by the previous round plus fresh ones, up to
 * B = or_maslov_round_size(M); every attempt of a round is evaluated on the
 * state the previous round left; a valid attempt claims its two slots and the
 * table entries of its two new pairs (lowest attempt index wins); attempts
 * owning all four commit (they touch disjoint slots and create distinct
 * pairs, so they commute); valid attempts that lost, and rejected attempts
 * whose reads a lower-index valid attempt may write (it claimed one of their
 * slots or checked pair entries, or commits the removal of a checked pair),
 * are deferred; the other rejected attempts are decided.  Every requested attempt is
 * evaluated once; the result is the GPU kernel's bit for bit. */
static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int64_t or_maslov_round_size(int64_t M);
int64_t or_maslov_round_size(int64_t M)
{
    int64_t b = M / 32;
    if (b < 64) b = 64;
    if (b > (1LL << 20)) b = 1LL << 20;
    return b;
}

static uint32_t maslov_table_size(int64_t B)
{
    uint32_t h = 1024;
    while ((int64_t)h < 64 * B) h <<= 1;
    return h;
}

/* Random bits q of the stream of `seed`: splitmix64 outputs at counter q of
 * a key derived from the seed, so streams of different seeds do not overlap
 * (a plain seed ^ q would make the streams of small seeds permutations of
 * one another). */
static inline uint64_t stream_key(uint64_t seed) { return mix64(seed ^ 0xD1B54A32D192ED03ULL); }
static inline uint64_t stream_bits(uint64_t key, uint64_t q) { return mix64(key + q * 0x9E3779B97F4A7C15ULL); }

static inline uint32_t pair_entry(int a, int b, int64_t N, uint32_t hmask)
{
    uint64_t lo = (uint64_t)(a < b ? a : b), hi = (uint64_t)(a < b ? b : a);
    return (uint32_t)(mix64(lo * (uint64_t)N + hi) & hmask);
}

static inline int has_edge(const uint64_t* bits, int64_t N, int a, int b)
{
    uint64_t q = (uint64_t)a * (uint64_t)N + (uint64_t)b;
    return (int)((bits[q >> 6] >> (q & 63)) & 1ULL);
}
static inline void set_edge(uint64_t* bits, int64_t N, int a, int b, int on)
{
    uint64_t q = (uint64_t)a * (uint64_t)N + (uint64_t)b;
    if (on) bits[q >> 6] |= 1ULL << (q & 63); else bits[q >> 6] &= ~(1ULL << (q & 63));
}

/* CSR of the rewired slots with ascending columns; each undirected slot's
 * weight goes to both directions (Maslov_weighted_1's vu/vl re-attachment,
 * W/Maslov/Maslov/Maslov.cpp:145-186); R is unchanged (degrees preserved). */
static void maslov_rebuild(const int32_t* R, int N, int64_t M, const int32_t* ea, const int32_t* eb,
                           const float* ew, int32_t* R_out, int32_t* C_out, float* V_out)
{
    int64_t* cur = (int64_t*)malloc((size_t)(N + 1) * sizeof(int64_t));
    for (int i = 0; i <= N; i++) R_out[i] = R[i];
    int32_t* tmpc = (int32_t*)malloc((size_t)(R[N] > 0 ? R[N] : 1) * sizeof(int32_t));
    float* tmpw = (float*)malloc((size_t)(R[N] > 0 ? R[N] : 1) * sizeof(float));
    for (int i = 0; i < N; i++) cur[i] = R[i];
    for (int64_t e = 0; e < M; e++) {
        int a = ea[e], b = eb[e];
        tmpc[cur[a]] = b; tmpw[cur[a]] = ew[e]; cur[a]++;
        tmpc[cur[b]] = a; tmpw[cur[b]] = ew[e]; cur[b]++;
    }
    /* sort each row by column (insertion sort is fine for oracle sizes) */
    for (int i = 0; i < N; i++) {
        for (int32_t x = R[i] + 1; x < R[i + 1]; x++) {
            int32_t c = tmpc[x]; float w = tmpw[x]; int32_t y = x - 1;
            while (y >= R[i] && tmpc[y] > c) { tmpc[y + 1] = tmpc[y]; tmpw[y + 1] = tmpw[y]; y--; }
            tmpc[y + 1] = c; tmpw[y + 1] = w;
        }
    }
    memcpy(C_out, tmpc, sizeof(int32_t) * (size_t)R[N]);
    if (V_out) memcpy(V_out, tmpw, sizeof(float) * (size_t)R[N]);
    free(tmpc); free(tmpw); free(cur);
}

typedef struct {
    uint64_t a;
    int v[4];
    int64_t i, j;
    uint32_t h[2];        /* table entries of the two new pairs */
    int state;            /* 0 shared end point, 1 new edge exists, 2 valid */
    int coin;
} MsItem;

int64_t or_maslov(const int32_t* R, const int32_t* C, const float* V, int N, uint64_t seed,
                  int64_t attempts, int32_t* R_out, int32_t* C_out, float* V_out)
{
    int64_t M = R[N] / 2;
    int32_t* ea = (int32_t*)malloc((size_t)(M > 0 ? M : 1) * sizeof(int32_t));
    int32_t* eb = (int32_t*)malloc((size_t)(M > 0 ? M : 1) * sizeof(int32_t));
    float* ew = (float*)malloc((size_t)(M > 0 ? M : 1) * sizeof(float));
    size_t words = (size_t)(((uint64_t)N * (uint64_t)N + 63) / 64);
    uint64_t* bits = (uint64_t*)calloc(words > 0 ? words : 1, sizeof(uint64_t));
    int64_t m = 0;
    for (int i = 0; i < N; i++)
        for (int32_t e = R[i]; e < R[i + 1]; e++) {
            set_edge(bits, N, i, C[e], 1);
            if (C[e] > i) { ea[m] = i; eb[m] = C[e]; ew[m] = V ? V[e] : 1.0f; m++; }
        }
    int64_t committed = 0;
    const int64_t B = or_maslov_round_size(M);
    const uint32_t H = maslov_table_size(B), hmask = H - 1;
    /* claims of valid attempts, then the writes of committed ones */
    uint64_t* slot_owner = (uint64_t*)malloc((size_t)(M > 0 ? M : 1) * sizeof(uint64_t));
    uint64_t* table = (uint64_t*)malloc((size_t)H * sizeof(uint64_t));
    uint64_t* pair_wr = (uint64_t*)malloc((size_t)H * sizeof(uint64_t));
    for (int64_t q = 0; q < M; q++) slot_owner[q] = UINT64_MAX;
    for (uint32_t q = 0; q < H; q++) table[q] = pair_wr[q] = UINT64_MAX;
    MsItem* items = (MsItem*)malloc((size_t)B * sizeof(MsItem));
    unsigned char* commit = (unsigned char*)malloc((size_t)B);
    uint64_t* pend = (uint64_t*)malloc((size_t)B * sizeof(uint64_t));
    uint64_t* pnext = (uint64_t*)malloc((size_t)B * sizeof(uint64_t));
    int64_t np = 0;
    uint64_t fresh = 0;
    const uint64_t key = stream_key(seed);
    while (M >= 2) {
        uint64_t left = (uint64_t)attempts - fresh;
        uint64_t take = left < (uint64_t)(B - np) ? left : (uint64_t)(B - np);
        int64_t total = np + (int64_t)take;
        if (total == 0) break;
        /* evaluate on the round's state; valid attempts claim */
        for (int64_t it = 0; it < total; it++) {
            MsItem* t = &items[it];
            t->a = it < np ? pend[it] : fresh + (uint64_t)(it - np);
            uint64_t h1 = stream_bits(key, 2 * t->a), h2 = stream_bits(key, 2 * t->a + 1);
            t->i = (int64_t)(h1 % (uint64_t)M);
            t->j = (int64_t)(h2 % (uint64_t)M);
            t->coin = (int)((h1 >> 63) ^ (h2 >> 63));
            t->v[0] = ea[t->i]; t->v[1] = eb[t->i]; t->v[2] = ea[t->j]; t->v[3] = eb[t->j];
            int x1 = t->v[0], x2 = t->coin ? t->v[2] : t->v[3];   /* 1-3 or 1-4 */
            int y1 = t->v[1], y2 = t->coin ? t->v[3] : t->v[2];   /* 2-4 or 2-3 */
            t->h[0] = pair_entry(x1, x2, N, hmask);
            t->h[1] = pair_entry(y1, y2, N, hmask);
            if (t->v[0] == t->v[2] || t->v[0] == t->v[3] || t->v[1] == t->v[2] || t->v[1] == t->v[3]) t->state = 0;
            else if (has_edge(bits, N, x1, x2) || has_edge(bits, N, y1, y2)) t->state = 1;
            else t->state = 2;
            if (t->state == 2) {
                if (slot_owner[t->i] > t->a) slot_owner[t->i] = t->a;
                if (slot_owner[t->j] > t->a) slot_owner[t->j] = t->a;
                if (table[t->h[0]] > t->a) table[t->h[0]] = t->a;
                if (table[t->h[1]] > t->a) table[t->h[1]] = t->a;
            }
        }
        /* valid attempts owning all four claims commit; they record the two
         * pairs they remove */
        for (int64_t it = 0; it < total; it++) {
            MsItem* t = &items[it];
            commit[it] = t->state == 2 && slot_owner[t->i] == t->a && slot_owner[t->j] == t->a &&
                         table[t->h[0]] == t->a && table[t->h[1]] == t->a;
            if (!commit[it]) continue;
            uint32_t w[2] = {pair_entry(t->v[0], t->v[1], N, hmask), pair_entry(t->v[2], t->v[3], N, hmask)};
            for (int q = 0; q < 2; q++) if (pair_wr[w[q]] > t->a) pair_wr[w[q]] = t->a;
        }
        /* apply the commits; every valid attempt that lost is deferred, and so
         * is a rejected attempt when a lower-index valid attempt claimed one of
         * its slots or a pair entry it checked, or a lower-index commit removes
         * a pair it checked (conservative: such an attempt may not commit) */
        int64_t nn = 0;
        for (int64_t it = 0; it < total; it++) {
            MsItem* t = &items[it];
            if (t->state == 2 && !commit[it]) { pnext[nn++] = t->a; continue; }
            if (t->state < 2) {
                int stale = slot_owner[t->i] < t->a || slot_owner[t->j] < t->a;
                if (t->state == 1)
                    stale |= table[t->h[0]] < t->a || table[t->h[1]] < t->a ||
                             pair_wr[t->h[0]] < t->a || pair_wr[t->h[1]] < t->a;
                if (stale) pnext[nn++] = t->a;
                continue;
            }
            int V1 = t->v[0], V2 = t->v[1], V3 = t->v[2], V4 = t->v[3];
            set_edge(bits, N, V1, V2, 0); set_edge(bits, N, V2, V1, 0);
            set_edge(bits, N, V3, V4, 0); set_edge(bits, N, V4, V3, 0);
            if (t->coin) {   /* 1-3, 2-4 (Maslov.cpp:36-44) */
                set_edge(bits, N, V1, V3, 1); set_edge(bits, N, V3, V1, 1);
                set_edge(bits, N, V2, V4, 1); set_edge(bits, N, V4, V2, 1);
                eb[t->i] = V3; ea[t->j] = V2;
            } else {         /* 1-4, 3-2 (Maslov.cpp:47-56) */
                set_edge(bits, N, V1, V4, 1); set_edge(bits, N, V4, V1, 1);
                set_edge(bits, N, V2, V3, 1); set_edge(bits, N, V3, V2, 1);
                eb[t->i] = V4; eb[t->j] = V2;
            }
            committed++;
        }
        for (int64_t it = 0; it < total; it++) {
            MsItem* t = &items[it];
            slot_owner[t->i] = slot_owner[t->j] = UINT64_MAX;
            table[t->h[0]] = table[t->h[1]] = pair_wr[t->h[0]] = pair_wr[t->h[1]] = UINT64_MAX;
            pair_wr[pair_entry(t->v[0], t->v[1], N, hmask)] = UINT64_MAX;
            pair_wr[pair_entry(t->v[2], t->v[3], N, hmask)] = UINT64_MAX;
        }
        uint64_t* tmp = pend; pend = pnext; pnext = tmp;
        np = nn;
        fresh += take;
    }
    free(slot_owner); free(table); free(pair_wr); free(items); free(commit); free(pend); free(pnext);
    maslov_rebuild(R, N, M, ea, eb, ew, R_out, C_out, V_out);
    free(ea); free(eb); free(ew); free(bits);
    return committed;
}

/* The reference's Rewire loop itself (U/cuda_EC/cuda_EC/Maslov.cpp:17-59,
 * W/Maslov/Maslov/Maslov.cpp:59-101), attempt after attempt on the current
 * graph, drawing from the 15-bit linear congruential rand() of the Microsoft
 * C runtime the reference was built with (state = state * 214013 + 2531011,
 * output bits 16..30) seeded with `seed` where the reference calls
 * srand(time(0)): slot i = (rand() * 0x8000 + rand()) % M, slot j likewise,
 * coin = rand() % 2.  Returns the number of committed swaps (the reference's
 * Shuffle_times).  With the stream of the reference's run this is the
 * reference's result exactly. */
int64_t or_rewire_seq(const int32_t* R, const int32_t* C, const float* V, int N, uint32_t seed, int64_t attempts,
                      int32_t* R_out, int32_t* C_out, float* V_out)
{
    int64_t M = R[N] / 2;
    int32_t* ea = (int32_t*)malloc((size_t)(M > 0 ? M : 1) * sizeof(int32_t));
    int32_t* eb = (int32_t*)malloc((size_t)(M > 0 ? M : 1) * sizeof(int32_t));
    float* ew = (float*)malloc((size_t)(M > 0 ? M : 1) * sizeof(float));
    size_t words = (size_t)(((uint64_t)N * (uint64_t)N + 63) / 64);
    uint64_t* bits = (uint64_t*)calloc(words > 0 ? words : 1, sizeof(uint64_t));
    int64_t m = 0;
    for (int i = 0; i < N; i++)
        for (int32_t e = R[i]; e < R[i + 1]; e++) {
            set_edge(bits, N, i, C[e], 1);
            if (C[e] > i) { ea[m] = i; eb[m] = C[e]; ew[m] = V ? V[e] : 1.0f; m++; }
        }
    uint32_t st = seed;
#define RAND15() (st = st * 214013u + 2531011u, (int)((st >> 16) & 0x7fff))
    int64_t committed = 0;
    for (int64_t k = 0; M > 0 && k < attempts; k++) {
        int hi = RAND15(), lo = RAND15();
        int64_t i = ((int64_t)hi * 0x8000 + lo) % M;
        hi = RAND15(); lo = RAND15();
        int64_t j = ((int64_t)hi * 0x8000 + lo) % M;
        int V1 = ea[i], V2 = eb[i], V3 = ea[j], V4 = eb[j];
        if (V1 == V3 || V1 == V4 || V2 == V3 || V2 == V4) continue;
        if (RAND15() % 2) {
            if (has_edge(bits, N, V1, V3) || has_edge(bits, N, V2, V4)) continue;
            set_edge(bits, N, V1, V2, 0); set_edge(bits, N, V2, V1, 0);
            set_edge(bits, N, V3, V4, 0); set_edge(bits, N, V4, V3, 0);
            set_edge(bits, N, V1, V3, 1); set_edge(bits, N, V3, V1, 1);
            set_edge(bits, N, V2, V4, 1); set_edge(bits, N, V4, V2, 1);
            eb[i] = V3; ea[j] = V2;
        } else {
            if (has_edge(bits, N, V1, V4) || has_edge(bits, N, V2, V3)) continue;
            set_edge(bits, N, V1, V2, 0); set_edge(bits, N, V2, V1, 0);
            set_edge(bits, N, V3, V4, 0); set_edge(bits, N, V4, V3, 0);
            set_edge(bits, N, V1, V4, 1); set_edge(bits, N, V4, V1, 1);
            set_edge(bits, N, V2, V3, 1); set_edge(bits, N, V3, V2, 1);
            eb[i] = V4; eb[j] = V2;
        }
        committed++;
    }
#undef RAND15
    maslov_rebuild(R, N, M, ea, eb, ew, R_out, C_out, V_out);
    free(ea); free(eb); free(ew); free(bits);
    return committed;
}

/* ------------------------------------------------- eigenvector centrality */
/* The power method of the two CUEC tools: Lead_Vector_GPU in
 * U/CUEC/CUEC/CUEC_unweighted.cu:61-214 (every edge value 1) and in
 * W/CUEC/weighted-net.cu:55-218 (the CSR weights as double).  u starts as the
 * node ids (init_AD, :38-43 in both files).  A step (:153-188 / :154-187):
 * u0 = u; vNorm = |u|; u = u * (1 / vNorm); y = A u; err1 = |y - u0|,
 * err2 = |y + u0|; the loop ends when either is at most 1e-6 or after 10,000
 * steps.  The unweighted tool keeps the normalised u of the last step
 * (:161), the weighted tool the last y (:190); both return vNorm as the
 * eigenvalue.  `raw` selects the weighted tool's output.  Norms are plain
 * sequential sums of squares (the reference's cuBLAS nrm2 is not vendored).
 * Returns the number of steps. */
int or_eigen_centrality(const int32_t* R, const int32_t* C, const float* V, int N, int raw,
                        double* ec, double* eigenvalue, double* residual)
{
    double* u = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    double* u0 = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    double* x = (double*)malloc(sizeof(double) * (size_t)(N > 0 ? N : 1));
    for (int i = 0; i < N; i++) u[i] = (double)i;
    double err1 = 1.0, err2 = 1.0, vnorm = 0.0;
    int iter = 0;
    while (err1 > 1e-6 && err2 > 1e-6 && iter < 10000) {
        for (int i = 0; i < N; i++) u0[i] = u[i];
        vnorm = nm_norm(u, N);
        const double inv = 1.0 / vnorm;
        for (int i = 0; i < N; i++) x[i] = u[i] * inv;
        for (int i = 0; i < N; i++) {
            double t = 0.0;
            for (int32_t j = R[i]; j < R[i + 1]; j++) t += (V ? (double)V[j] : 1.0) * x[C[j]];
            u[i] = t;
        }
        double s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < N; i++) {
            const double d1 = u[i] - u0[i], d2 = u[i] + u0[i];
            s1 += d1 * d1;
            s2 += d2 * d2;
        }
        err1 = sqrt(s1);
        err2 = sqrt(s2);
        iter++;
    }
    for (int i = 0; i < N; i++) ec[i] = raw ? u[i] : x[i];
    if (eigenvalue) *eigenvalue = vnorm;
    if (residual) *residual = err1 < err2 ? err1 : err2;
    free(u); free(u0); free(x);
    return iter;
}

/* --------------------------------------------- participation coefficient */
/* PC_CPU (W/PC_CPU/PC_CPU/main.cpp:100-174), float arithmetic in the same
 * order: strength s_i = sum of the row's weights (row order), per-module
 * weight sums in row order, PC_i = 1 - sum_m (w_im / s_i)^2 over modules
 * 1..K in order (0 when s_i = 0); normalised = PC / ((K-1)/K) unless K = 1.
 * module: float labels 1..K per node (the _modu.nm file).  V null: weight 1.
 * Labels below 1 are skipped (the reference would write outside its array). */
int or_participation(const int32_t* R, const int32_t* C, const float* V, int N, const float* module,
                     float* pc, float* pc_norm)
{
    int K = 0;
    for (int i = 0; i < N; i++)
        if ((int)module[i] > K) K = (int)module[i];
    float* within = (float*)calloc((size_t)(K > 0 ? K : 1), sizeof(float));
    for (int i = 0; i < N; i++) {
        float deg = 0.0f;
        for (int32_t j = R[i]; j < R[i + 1]; j++) deg += V ? V[j] : 1.0f;
        if (deg == 0.0f) {
            pc[i] = 0.0f;
            continue;
        }
        memset(within, 0, sizeof(float) * (size_t)(K > 0 ? K : 1));
        for (int32_t j = R[i]; j < R[i + 1]; j++) {
            const int m = (int)module[C[j]];
            if (m >= 1) within[m - 1] += V ? V[j] : 1.0f;
        }
        float sum = 0.0f;
        for (int m = 0; m < K; m++) {
            const float t = within[m] / deg;
            sum += t * t;
        }
        pc[i] = 1.0f - sum;
    }
    const float mx = K != 1 ? (float)(K - 1) / (float)K : 1.0f;
    for (int i = 0; i < N; i++) pc_norm[i] = K != 1 ? pc[i] / mx : pc[i];
    free(within);
    return K;
}
