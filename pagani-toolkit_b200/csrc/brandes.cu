// brandes.cu -- Brandes betweenness from all sources (CUBC, U/BC/CUBC/
// BC_GPU_node_pred.cu:6-155; Betweenness_CPU, U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:6-82)
// with exact 64-bit path counts and FP64 dependencies.
//
// 32 sources run together, one warp lane per source: per node the state is
// a row of 32 entries (level int32, sigma uint64, coefficient double), so a
// neighbour's state for all sources is one coalesced 128/256-byte read.
// Source bits of the current frontier are a 32-bit mask per node.
//   forward level d:  v finds the sources that reach it at d (OR of the
//                     frontier masks of its neighbours), then sums
//                     sigma[u][s] over neighbours u on level d-1 of source s;
//   backward level d: v on level d of source s sums
//                     (1 + delta[w][s]) / sigma[w][s] over neighbours w on
//                     level d+1 (kept as one coefficient per entry), so
//                     delta[v][s] = sigma[v][s] * sum; BC[v] += sum_s delta.
// BC[v] is the sum over ORDERED (source, target) pairs like the reference.
// The whole sweep over all source batches is one cooperative kernel; levels
// are separated by grid-wide barriers, so no host round trip happens per
// level.  The same forward pass yields the hop path length (sum of 1/d per
// node), which pg_betweenness can return as well.
#include "pg_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>

namespace cg = cooperative_groups;

namespace {
constexpr int THREADS = 256;
constexpr int LCAP = 48;      // levels whose frontier masks are kept for the backward sweep

struct BCArgs {
    const int32_t* R;
    const int32_t* C;
    int32_t n;
    const int32_t* sources;   // null: sources 0..n-1
    int32_t nsrc;
    int32_t* dist;            // [n][32]
    unsigned long long* sigma;  // [n][32]
    double* coef;             // [n][32]
    unsigned int* front;      // [2][n]
    unsigned int* fhist;      // [LCAP][n] frontier mask of every level < LCAP
    unsigned int* seen;       // [n]
    int* flags;               // [3] rotating "something changed" flags
    double* bc;               // [n] accumulated FP64 betweenness (null: forward only)
    double* inv;              // [n] sum of 1/d (null: skip)
    int do_backward;
    // pg_bfs_sigma output of one batch (null otherwise)
    int32_t* out_dist;
    unsigned long long* out_sigma;
};

__global__ void __launch_bounds__(THREADS)
k_brandes(BCArgs a, int batch_first, int batch_last)
{
    cg::grid_group grid = cg::this_grid();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int n = a.n;
    const size_t gt = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
    for (int b = batch_first; b < batch_last; b++) {
        const int s0 = b * 32;
        const int ns = min(32, a.nsrc - s0);
        const unsigned full = ns == 32 ? 0xffffffffu : ((1u << ns) - 1u);
        // ---- init: levels -1, frontier = sources
        for (size_t q = gt; q < (size_t)n * 32; q += gstride) a.dist[q] = -1;
        for (size_t v = gt; v < (size_t)n; v += gstride) { a.front[v] = 0u; a.seen[v] = 0u; a.fhist[v] = 0u; }
        if (gt < 3) a.flags[gt] = 0;
        grid.sync();
        if (gt < (size_t)ns) {
            int s = a.sources ? a.sources[s0 + gt] : s0 + (int)gt;
            a.dist[(size_t)s * 32 + gt] = 0;
            a.sigma[(size_t)s * 32 + gt] = 1ULL;
            atomicOr(&a.front[s], 1u << gt);
            atomicOr(&a.seen[s], 1u << gt);
            atomicOr(&a.fhist[s], 1u << gt);
        }
        grid.sync();
        // ---- forward
        int d = 1;
        unsigned int* cur = a.front;
        unsigned int* nxt = a.front + n;
        for (;; d++) {
            if (gt == 0) a.flags[(d + 1) % 3] = 0;
            int found = 0;
            for (int v = gw; v < n; v += nw) {
                const unsigned sv = a.seen[v];
                const unsigned need = full & ~sv;
                unsigned nb = 0;
                const int32_t s = a.R[v], e = a.R[v + 1];
                if (need) {
                    unsigned acc = 0;
                    for (int32_t base = s; base < e; base += 32) {
                        int32_t f = base + lane;
                        if (f < e) acc |= cur[a.C[f]];
                        acc = __reduce_or_sync(0xffffffffu, acc);
                        if ((acc & need) == need) break;
                    }
                    nb = acc & need;
                }
                if (nb) {
                    unsigned long long sg = 0;
                    for (int32_t base = s; base < e; base += 32) {
                        int32_t f = base + lane;
                        int u = f < e ? a.C[f] : 0;
                        unsigned fu = f < e ? (cur[u] & nb) : 0u;
                        unsigned m = __ballot_sync(0xffffffffu, fu != 0u);
                        while (m) {
                            int j = __ffs(m) - 1;
                            m &= m - 1;
                            int uj = __shfl_sync(0xffffffffu, u, j);
                            unsigned fj = __shfl_sync(0xffffffffu, fu, j);
                            if ((fj >> lane) & 1u) sg += a.sigma[(size_t)uj * 32 + lane];
                        }
                    }
                    if ((nb >> lane) & 1u) {
                        a.sigma[(size_t)v * 32 + lane] = sg;
                        a.dist[(size_t)v * 32 + lane] = d;
                    }
                    if (lane == 0 && a.inv) a.inv[v] += (double)__popc(nb) / (double)d;
                    found = 1;
                }
                if (lane == 0) {
                    nxt[v] = nb;
                    a.seen[v] = sv | nb;
                    if (d < LCAP) a.fhist[(size_t)d * n + v] = nb;
                }
            }
            if (found && lane == 0) a.flags[d % 3] = 1;
            grid.sync();
            const int any = a.flags[d % 3];
            unsigned int* t = cur; cur = nxt; nxt = t;
            if (!any) break;
        }
        const int maxd = d - 1;  // deepest level reached
        if (a.out_dist) {
            for (size_t q = gt; q < (size_t)ns * n; q += gstride) {
                size_t sidx = q / n, v = q % n;
                a.out_dist[q] = a.dist[v * 32 + sidx];
                a.out_sigma[q] = a.dist[v * 32 + sidx] >= 0 ? a.sigma[v * 32 + sidx] : 0ULL;
            }
        }
        // ---- backward
        if (a.do_backward) {
            for (int lv = maxd; lv >= 1; lv--) {
                for (int v = gw; v < n; v += nw) {
                    // sources for which v sits on level lv
                    unsigned mine_m;
                    if (lv < LCAP) mine_m = a.fhist[(size_t)lv * n + v];
                    else mine_m = __ballot_sync(0xffffffffu, a.dist[(size_t)v * 32 + lane] == lv);
                    if (!mine_m) continue;
                    const bool mine = (mine_m >> lane) & 1u;
                    double acc = 0.0;
                    if (lv < maxd) {
                        const int32_t s = a.R[v], e = a.R[v + 1];
                        for (int32_t base = s; base < e; base += 32) {
                            int32_t f = base + lane;
                            int w = f < e ? a.C[f] : 0;
                            if (lv + 1 < LCAP) {
                                // neighbours one level deeper for some of v's sources
                                unsigned mw = f < e ? (a.fhist[(size_t)(lv + 1) * n + w] & mine_m) : 0u;
                                unsigned bm = __ballot_sync(0xffffffffu, mw != 0u);
                                while (bm) {
                                    int j = __ffs(bm) - 1;
                                    bm &= bm - 1;
                                    int wj = __shfl_sync(0xffffffffu, w, j);
                                    unsigned mj = __shfl_sync(0xffffffffu, mw, j);
                                    if ((mj >> lane) & 1u) acc += a.coef[(size_t)wj * 32 + lane];
                                }
                            } else {
                                int cnt = min(32, e - base);
                                for (int j = 0; j < cnt; j++) {
                                    int wj = __shfl_sync(0xffffffffu, w, j);
                                    int dw = a.dist[(size_t)wj * 32 + lane];
                                    if (mine && dw == lv + 1) acc += a.coef[(size_t)wj * 32 + lane];
                                }
                            }
                        }
                    }
                    double delta = 0.0;
                    if (mine) {
                        double sg = __ull2double_rn(a.sigma[(size_t)v * 32 + lane]);
                        delta = sg * acc;
                        a.coef[(size_t)v * 32 + lane] = (1.0 + delta) / sg;
                    }
                    double tot = delta;
                    for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
                    if (lane == 0 && a.bc) a.bc[v] += tot;
                }
                grid.sync();
            }
        }
        grid.sync();
    }
}

__global__ void k_bc_out(const double* __restrict__ bc, const double* __restrict__ inv, int32_t n,
                         float* __restrict__ bcf, float* __restrict__ eff)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (bcf) bcf[v] = (float)bc[v];
        if (eff) eff[v] = n > 1 ? (float)(inv[v] / (double)(n - 1)) : 0.0f;
    }
}

__global__ void k_sum_inv(const double* __restrict__ x, int32_t n, double* __restrict__ out)
{
    __shared__ double sh[1024];
    double acc = 0.0;
    int per = (n + blockDim.x - 1) / blockDim.x;
    int lo = threadIdx.x * per, hi = min(n, lo + per);
    for (int i = lo; i < hi; i++) acc += x[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)blockDim.x; i++) t += sh[i];
        *out = t;
    }
}

pg_status alloc_state(pg_ctx* ctx, int n, BCArgs& a)
{
    PG_TRY(pg_wst(ctx, "bc.dist", (size_t)n * 32 + 32, &a.dist));
    PG_TRY(pg_wst(ctx, "bc.sigma", (size_t)n * 32 + 32, &a.sigma));
    PG_TRY(pg_wst(ctx, "bc.coef", (size_t)n * 32 + 32, &a.coef));
    PG_TRY(pg_wst(ctx, "bc.front", (size_t)2 * n + 2, &a.front));
    PG_TRY(pg_wst(ctx, "bc.fhist", (size_t)LCAP * n + 2, &a.fhist));
    PG_TRY(pg_wst(ctx, "bc.seen", (size_t)n + 1, &a.seen));
    PG_TRY(pg_wst(ctx, "bc.flags", 4, &a.flags));
    return PG_OK;
}

pg_status launch_brandes(pg_ctx* ctx, BCArgs& a, int batch_first, int batch_last)
{
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_brandes, THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "brandes kernel cannot be resident");
    int grid = per_sm * ctx->sm_count;
    void* args[] = {(void*)&a, (void*)&batch_first, (void*)&batch_last};
    PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_brandes, dim3(grid), dim3(THREADS), args, 0, ctx->stream));
    PG_LAUNCHED(ctx);
    return PG_OK;
}
}  // namespace

extern "C" pg_status pg_betweenness(pg_ctx* ctx, const pg_graph* g, float* bc, double* bc64, float* eff, double* lp)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_betweenness: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    BCArgs a = {};
    a.R = g->R;
    a.C = g->C;
    a.n = n;
    a.nsrc = n;
    a.do_backward = 1;
    PG_TRY(alloc_state(ctx, n, a));
    PG_TRY(pg_wst(ctx, "bc.bc", (size_t)n + 1, &a.bc));
    PG_CUDA(ctx, cudaMemsetAsync(a.bc, 0, sizeof(double) * (n + 1), ctx->stream));
    if (eff || lp) {
        PG_TRY(pg_wst(ctx, "bc.inv", (size_t)n + 1, &a.inv));
        PG_CUDA(ctx, cudaMemsetAsync(a.inv, 0, sizeof(double) * (n + 1), ctx->stream));
    }
    const int nb = (n + 31) / 32;
    // a few batches per launch keeps every launch short
    const int per_launch = 64;
    for (int b = 0; b < nb; b += per_launch) PG_TRY(launch_brandes(ctx, a, b, std::min(nb, b + per_launch)));
    float *dbc, *deff = nullptr;
    PG_TRY(pg_wst(ctx, "bc.bcf", (size_t)n + 1, &dbc));
    if (eff) PG_TRY(pg_wst(ctx, "bc.eff", (size_t)n + 1, &deff));
    k_bc_out<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(a.bc, a.inv, n, dbc, deff);
    PG_LAUNCHED(ctx);
    if (bc) PG_TRY(pg_d2h(ctx, bc, dbc, sizeof(float) * n));
    if (bc64) PG_TRY(pg_d2h(ctx, bc64, a.bc, sizeof(double) * n));
    if (eff) PG_TRY(pg_d2h(ctx, eff, deff, sizeof(float) * n));
    if (lp) {
        double* tot;
        PG_TRY(pg_wst(ctx, "bc.tot", 1, &tot));
        k_sum_inv<<<1, 1024, 0, ctx->stream>>>(a.inv, n, tot);
        PG_LAUNCHED(ctx);
        double t;
        PG_TRY(pg_d2h(ctx, &t, tot, sizeof t));
        *lp = t > 0.0 ? (double)n * (double)(n - 1) / t : 0.0;
    }
    return PG_OK;
}

extern "C" pg_status pg_bfs_sigma(pg_ctx* ctx, const pg_graph* g, const int32_t* sources, int32_t ns, int32_t* dist,
                                  int64_t* sigma)
{
    if (!ctx || !g || !sources || ns < 0 || !dist || !sigma)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_bfs_sigma: bad arguments");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    for (int i = 0; i < ns; i++)
        if (sources[i] < 0 || sources[i] >= n) return pg_fail(ctx, PG_ERR_INVALID, "source %d out of range", sources[i]);
    BCArgs a = {};
    a.R = g->R;
    a.C = g->C;
    a.n = n;
    a.nsrc = ns;
    PG_TRY(alloc_state(ctx, n, a));
    int32_t* dsrc;
    PG_TRY(pg_wst(ctx, "bc.src", (size_t)ns + 1, &dsrc));
    PG_CUDA(ctx, cudaMemcpyAsync(dsrc, sources, sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream));
    a.sources = dsrc;
    PG_TRY(pg_wst(ctx, "bc.odist", (size_t)32 * n, &a.out_dist));
    PG_TRY(pg_wst(ctx, "bc.osigma", (size_t)32 * n, &a.out_sigma));
    for (int b = 0; b < (ns + 31) / 32; b++) {
        PG_TRY(launch_brandes(ctx, a, b, b + 1));
        int cnt = std::min(32, ns - b * 32);
        PG_TRY(pg_d2h(ctx, dist + (size_t)b * 32 * n, a.out_dist, sizeof(int32_t) * (size_t)cnt * n));
        PG_TRY(pg_d2h(ctx, sigma + (size_t)b * 32 * n, a.out_sigma, sizeof(int64_t) * (size_t)cnt * n));
    }
    return PG_OK;
}
