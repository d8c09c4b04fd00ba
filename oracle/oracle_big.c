/*
 * oracle_big.c -- the checker's restatements at subject size (tens of
 * thousands of voxels), where the packed matrix of oracle.c (M1 doubles) and
 * its single-thread loops no longer fit a few minutes.  TEST INFRASTRUCTURE
 * ONLY: used by tests/golden/make_subject58k.py to write fixtures, and by the
 * CPU tests that pin these functions to oracle.c on small inputs.  The
 * product library never links it.
 *
 * Results are those of oracle.c, not approximations of them:
 *   - or_big_topk restates select + FormFullGraph_s
 *     (U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:655-773) on the r of
 *     or_pair_r: every r is the same fma() chain over t ascending (a vector
 *     lane's fused multiply-add rounds once, exactly as the scalar fma()), the
 *     same range rule (CorMat.cpp:821) and key (r or |r|); the pairs are
 *     returned in (key descending, i ascending, j ascending) order, so the
 *     first k of them are the reference's selection for k edges: every key
 *     above the k-th, then the lexicographically first ties (:748-759);
 *   - or_brandes_mt is or_brandes (U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:6-82, int64
 *     sigma, FP64 delta) with the sources split over threads; each thread
 *     sums its own sources and the partial sums are added in thread order,
 *     so only the order of the FP64 additions into BC differs.
 *
 * Build (oracle/Makefile, target big): gcc -O2 -mavx2 -mfma
 * -ffp-contract=off -pthread; only the intrinsics below fuse.
 */
#include <immintrin.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ pair keys */
#define HBITS 20
#define HBINS (1 << HBITS)

typedef struct {
    const double* zt;      /* T x Np, column j of time t at zt[t*Np + j] */
    const double* z;       /* N x T row-major */
    int N, Np, T, abs_mode, weighted;
} Pairs;

static inline double range_rule(double r, int weighted)
{
    if (weighted) return (r > -1.0 - 1e-6 && r < 1.0 + 1e-6) ? r : 0.0;
    return (r >= -1.0 && r <= 1.0) ? r : 0.0;
}

static inline double key_of(double r, const Pairs* P)
{
    r = range_rule(r, P->weighted);
    return P->abs_mode ? fabs(r) : r;
}

/* order-preserving image of a double in the unsigned integers */
static inline uint64_t ord64(double x)
{
    uint64_t u;
    memcpy(&u, &x, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}

/* r of rows i0..i0+3 (rows past N-1 ignored) against the 12 columns
 * j0..j0+11, each as fma(z_i[t], z_j[t], acc) over t ascending. */
static inline void tile_4x12(const Pairs* P, int i0, int j0, double out[4][12])
{
    __m256d acc[4][3];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 3; b++) acc[a][b] = _mm256_setzero_pd();
    const double* zi[4];
    for (int a = 0; a < 4; a++) {
        int i = i0 + a < P->N ? i0 + a : P->N - 1;
        zi[a] = P->z + (int64_t)i * P->T;
    }
    for (int t = 0; t < P->T; t++) {
        const double* col = P->zt + (int64_t)t * P->Np + j0;
        __m256d c0 = _mm256_loadu_pd(col), c1 = _mm256_loadu_pd(col + 4), c2 = _mm256_loadu_pd(col + 8);
        for (int a = 0; a < 4; a++) {
            __m256d x = _mm256_broadcast_sd(zi[a] + t);
            acc[a][0] = _mm256_fmadd_pd(x, c0, acc[a][0]);
            acc[a][1] = _mm256_fmadd_pd(x, c1, acc[a][1]);
            acc[a][2] = _mm256_fmadd_pd(x, c2, acc[a][2]);
        }
    }
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 3; b++) _mm256_storeu_pd(&out[a][b * 4], acc[a][b]);
}

typedef struct {
    const Pairs* P;
    int* next_block;        /* shared: next block of 4 rows */
    pthread_mutex_t* mu;
    int64_t* hist;          /* pass 1: HBINS counts (per thread) */
    uint64_t floor_ord;     /* pass 2: keep keys with ord64 >= floor_ord */
    double* keys;           /* pass 2: per-thread output */
    int32_t *ii, *jj;
    int64_t n, cap;
    int pass, failed;
} Work;

static int take_block(Work* w)
{
    pthread_mutex_lock(w->mu);
    int b = (*w->next_block)++;
    pthread_mutex_unlock(w->mu);
    return b;
}

static void emit(Work* w, double key, int i, int j)
{
    if (w->n == w->cap) {
        int64_t cap = w->cap ? w->cap * 2 : (1 << 20);
        double* k2 = (double*)realloc(w->keys, (size_t)cap * sizeof(double));
        int32_t* i2 = k2 ? (int32_t*)realloc(w->ii, (size_t)cap * sizeof(int32_t)) : NULL;
        int32_t* j2 = i2 ? (int32_t*)realloc(w->jj, (size_t)cap * sizeof(int32_t)) : NULL;
        if (!k2 || !i2 || !j2) { w->failed = 1; return; }
        w->keys = k2; w->ii = i2; w->jj = j2; w->cap = cap;
    }
    w->keys[w->n] = key;
    w->ii[w->n] = i;
    w->jj[w->n] = j;
    w->n++;
}

static void* pair_worker(void* arg)
{
    Work* w = (Work*)arg;
    const Pairs* P = w->P;
    double out[4][12];
    for (;;) {
        int i0 = take_block(w) * 4;
        if (i0 >= P->N - 1) break;
        int jstart = (i0 + 1) / 4 * 4;
        for (int j0 = jstart; j0 < P->N; j0 += 12) {
            tile_4x12(P, i0, j0, out);
            for (int a = 0; a < 4; a++) {
                int i = i0 + a;
                if (i >= P->N) break;
                for (int b = 0; b < 12; b++) {
                    int j = j0 + b;
                    if (j <= i || j >= P->N) continue;
                    double key = key_of(out[a][b], P);
                    uint64_t o = ord64(key);
                    if (w->pass == 1) w->hist[o >> (64 - HBITS)]++;
                    else if (o >= w->floor_ord) emit(w, key, i, j);
                }
            }
        }
    }
    return NULL;
}

static int run_pass(Pairs* P, int threads, int pass, uint64_t floor_ord, Work* ws)
{
    int next = 0;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) {
        ws[t].P = P;
        ws[t].next_block = &next;
        ws[t].mu = &mu;
        ws[t].pass = pass;
        ws[t].floor_ord = floor_ord;
        pthread_create(&th[t], NULL, pair_worker, &ws[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(th);
    for (int t = 0; t < threads; t++)
        if (ws[t].failed) return -1;
    return 0;
}

typedef struct { double key; int32_t i, j; } Sel;

static int cmp_sel(const void* a, const void* b)
{
    const Sel* x = (const Sel*)a;
    const Sel* y = (const Sel*)b;
    if (x->key != y->key) return x->key < y->key ? 1 : -1;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    return (x->j > y->j) - (x->j < y->j);
}

/* The kmax pairs of largest key, in (key desc, i asc, j asc) order.  z is the
 * N x T FP64 z-score matrix of or_zscore.  Returns the number of pairs
 * written (min(kmax, M1)), or -1 when memory runs out. */
int64_t or_big_topk(const double* z, int N, int T, int abs_mode, int weighted, int64_t kmax, int threads,
                    double* key_out, int32_t* i_out, int32_t* j_out)
{
    int64_t M1 = (int64_t)N * (N - 1) / 2;
    if (kmax > M1) kmax = M1;
    if (kmax <= 0 || N < 2) return 0;
    if (threads < 1) threads = 1;
    Pairs P = {0};
    P.N = N;
    P.Np = (N + 11) / 12 * 12 + 12;
    P.T = T;
    P.abs_mode = abs_mode;
    P.weighted = weighted;
    P.z = z;
    double* zt = (double*)calloc((size_t)T * P.Np, sizeof(double));
    if (!zt) return -1;
    for (int i = 0; i < N; i++)
        for (int t = 0; t < T; t++) zt[(int64_t)t * P.Np + i] = z[(int64_t)i * T + t];
    P.zt = zt;

    Work* ws = (Work*)calloc((size_t)threads, sizeof(Work));
    for (int t = 0; t < threads; t++) ws[t].hist = (int64_t*)calloc(HBINS, sizeof(int64_t));
    run_pass(&P, threads, 1, 0, ws);
    int64_t* hist = ws[0].hist;
    for (int t = 1; t < threads; t++) {
        for (int b = 0; b < HBINS; b++) hist[b] += ws[t].hist[b];
        free(ws[t].hist);
        ws[t].hist = NULL;
    }
    /* the bin holding the kmax-th largest key: collect every key from it up */
    int64_t above = 0;
    int bstar = HBINS - 1;
    for (; bstar >= 0; bstar--) {
        if (above + hist[bstar] >= kmax) break;
        above += hist[bstar];
    }
    if (bstar < 0) bstar = 0;
    free(hist);
    ws[0].hist = NULL;
    uint64_t floor_ord = (uint64_t)bstar << (64 - HBITS);
    int rc = run_pass(&P, threads, 2, floor_ord, ws);
    free(zt);
    int64_t total = 0;
    for (int t = 0; t < threads; t++) total += ws[t].n;
    Sel* sel = rc == 0 ? (Sel*)malloc((size_t)(total > 0 ? total : 1) * sizeof(Sel)) : NULL;
    int64_t q = 0;
    for (int t = 0; t < threads; t++) {
        for (int64_t e = 0; sel && e < ws[t].n; e++, q++) {
            sel[q].key = ws[t].keys[e];
            sel[q].i = ws[t].ii[e];
            sel[q].j = ws[t].jj[e];
        }
        free(ws[t].keys); free(ws[t].ii); free(ws[t].jj);
    }
    free(ws);
    if (!sel) return -1;
    qsort(sel, (size_t)total, sizeof(Sel), cmp_sel);
    int64_t out = total < kmax ? total : kmax;
    for (int64_t e = 0; e < out; e++) {
        key_out[e] = sel[e].key;
        i_out[e] = sel[e].i;
        j_out[e] = sel[e].j;
    }
    free(sel);
    return out;
}

/* ----------------------------------------------------------- betweenness */
typedef struct {
    const int32_t *R, *C;
    int N, tid, threads;
    double* bc;
    double* inv_sum;        /* per source: sum over reached v of 1/d(s, v), or NULL */
} BcWork;

static void* brandes_worker(void* arg)
{
    BcWork* w = (BcWork*)arg;
    const int N = w->N;
    const int32_t *R = w->R, *C = w->C;
    int32_t* dist = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    int64_t* sigma = (int64_t*)malloc((size_t)N * sizeof(int64_t));
    double* delta = (double*)malloc((size_t)N * sizeof(double));
    int32_t* order = (int32_t*)malloc((size_t)N * sizeof(int32_t));
    for (int i = 0; i < N; i++) { dist[i] = -1; sigma[i] = 0; delta[i] = 0.0; }
    for (int s = w->tid; s < N; s += w->threads) {
        int head = 0, tail = 0;
        dist[s] = 0; sigma[s] = 1; order[tail++] = s;
        while (head < tail) {
            int v = order[head++];
            for (int32_t e = R[v]; e < R[v + 1]; e++) {
                int x = C[e];
                if (dist[x] < 0) { dist[x] = dist[v] + 1; order[tail++] = x; }
                if (dist[x] == dist[v] + 1) sigma[x] += sigma[v];
            }
        }
        if (w->inv_sum) {     /* the BFS order is by distance: sum count_d / d, d ascending */
            double acc = 0.0;
            int p = 1;
            while (p < tail) {
                int d = dist[order[p]], c = 0;
                while (p < tail && dist[order[p]] == d) { c++; p++; }
                acc += (double)c / d;
            }
            w->inv_sum[s] = acc;
        }
        for (int p = tail - 1; p >= 0; p--) {
            int x = order[p];
            double acc = 0.0;
            for (int32_t e = R[x]; e < R[x + 1]; e++) {
                int v = C[e];
                if (dist[v] == dist[x] + 1) acc += (1.0 + delta[v]) / (double)sigma[v];
            }
            delta[x] = (double)sigma[x] * acc;
            if (x != s) w->bc[x] += delta[x];
        }
        for (int p = 0; p < tail; p++) {      /* reset only what this source touched */
            int x = order[p];
            dist[x] = -1; sigma[x] = 0; delta[x] = 0.0;
        }
    }
    free(dist); free(sigma); free(delta); free(order);
    return NULL;
}

/* inv_sum (optional): per source s, sum_v 1/d(s, v) accumulated as
 * sum_d count_d / d with d ascending, as or_bfs_paths. */
void or_brandes_mt(const int32_t* R, const int32_t* C, int N, int threads, double* bc, double* inv_sum)
{
    if (threads < 1) threads = 1;
    BcWork* ws = (BcWork*)calloc((size_t)threads, sizeof(BcWork));
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) {
        ws[t] = (BcWork){R, C, N, t, threads, (double*)calloc((size_t)N, sizeof(double)), inv_sum};
        pthread_create(&th[t], NULL, brandes_worker, &ws[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    for (int i = 0; i < N; i++) {
        double s = 0.0;
        for (int t = 0; t < threads; t++) s += ws[t].bc[i];
        bc[i] = s;
    }
    for (int t = 0; t < threads; t++) free(ws[t].bc);
    free(ws);
    free(th);
}
