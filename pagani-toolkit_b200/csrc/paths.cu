// paths.cu -- hop path length and nodal efficiency (APSP_BFS,
// U/BFS_MulCPU/BFS_MulCPU/APSP_BFS.cpp:27-147) by bit-parallel multi-source
// BFS: 64*NW sources run together, one bit per source in NW 64-bit words per
// node.  Level 1 is a push from the batch's sources; every later level is a
// pull sweep: node v ORs the frontier words of its neighbours, keeps the
// bits it has not seen, and stops scanning once every missing source bit is
// found (tested every 128 neighbours).  Because the graph is undirected,
// d(s, v) = d(v, s), so node v counts the sources it reaches at each
// distance itself: cnt[v][d] (exact integers, summed over all batches), and
// at the end inv[v] = sum_d cnt[v][d] / d with d ascending -- the oracle's and
// APSP_BFS's per-source order, so the result does not depend on how the
// sources are batched and equals the oracle's bit for bit.  Distances beyond
// MAX_D are added to inv[v] directly as they are found.
//
// One cooperative launch runs every batch and level (grid-wide barriers
// between levels, the "any source still growing" flag in device memory), so
// the computation needs no host round trip and can be captured in a CUDA
// graph.  The sources per batch (NW) and the CTAs per SM are picked by the
// autotuner; the result is the same for every choice.
#include "pg_internal.cuh"
#include "paths.cuh"
#include "tune.cuh"
#include <algorithm>
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace {
constexpr int THREADS = 256;

template <int NW>
struct Words {
    unsigned long long w[NW];
};

template <int NW>
__global__ void __launch_bounds__(THREADS)
k_msbfs_all(PathArgs p)
{
    cg::grid_group grid = cg::this_grid();
    const int n = p.n;
    const int lane = threadIdx.x & 31;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    const int gw = (int)(tid >> 5), nw = (int)(nt >> 5);
    Words<NW>* front = (Words<NW>*)p.front;
    Words<NW>* next = (Words<NW>*)p.next;
    Words<NW>* seen_a = (Words<NW>*)p.seen_a;
    Words<NW>* seen_b = (Words<NW>*)p.seen_b;
    constexpr int SRC = 64 * NW;
    int diam = 0;
    for (int s0 = 0; s0 < n; s0 += SRC) {
        const int ns = min(SRC, n - s0);
        Words<NW> full;
#pragma unroll
        for (int q = 0; q < NW; q++) {
            const int c = max(0, min(64, ns - q * 64));
            full.w[q] = c == 64 ? ~0ULL : (c ? ((1ULL << c) - 1ULL) : 0ULL);
        }
        // level 1 by push: the batch's sources OR their bit into their
        // neighbours' frontier words (a pull sweep would read every edge)
        for (int v = (int)tid; v < n; v += (int)nt) {
            Words<NW> f, z;
#pragma unroll
            for (int q = 0; q < NW; q++) f.w[q] = z.w[q] = 0ULL;
            const int b = v - s0;
            if (b >= 0 && b < ns) f.w[b >> 6] = 1ULL << (b & 63);
            front[v] = z;
            seen_a[v] = f;
        }
        if (tid == 0) p.flags[0] = p.flags[1] = p.flags[2] = 0;
        grid.sync();
        for (int b = gw; b < ns; b += nw) {
            const int src = s0 + b;
            const unsigned long long bit = 1ULL << (b & 63);
            for (int32_t q = p.R[src] + lane; q < p.R[src + 1]; q += 32) atomicOr(&front[p.C[q]].w[b >> 6], bit);
        }
        grid.sync();
        {
            unsigned long long found_total = 0;
            for (int v = (int)tid; v < n; v += (int)nt) {
                const Words<NW> f = front[v], sv = seen_a[v];
                Words<NW> so;
                int cnt = 0;
#pragma unroll
                for (int q = 0; q < NW; q++) {
                    so.w[q] = sv.w[q] | f.w[q];
                    cnt += __popcll(f.w[q]);
                }
                seen_b[v] = so;
                if (cnt) p.cnt[(long long)v * MAX_D] += (unsigned)cnt;
                found_total += (unsigned)cnt;
            }
            for (int o = 16; o; o >>= 1) found_total += __shfl_xor_sync(0xffffffffu, found_total, o);
            if (lane == 0 && found_total && p.hist && 1 <= p.max_hop) atomicAdd(&p.hist[1], found_total);
            // one store per CTA: a store per warp to the same flag serialised in L2
            if (__syncthreads_or(found_total != 0) && threadIdx.x == 0) p.flags[1] = 1;
        }
        grid.sync();
        if (tid == 0) p.flags[0] = 0;
        if (!((volatile int*)p.flags)[1]) continue;   // no source has a neighbour
        diam = max(diam, 1);
        Words<NW>*sin = seen_b, *sout = seen_a, *cur = front, *nxt = next;
        for (int d = 2;; d++) {
            unsigned long long found_total = 0;
            for (int v = gw; v < n; v += nw) {
                const Words<NW> sv = sin[v];
                Words<NW> need, acc;
                bool any_need = false;
#pragma unroll
                for (int q = 0; q < NW; q++) {
                    need.w[q] = full.w[q] & ~sv.w[q];
                    any_need |= need.w[q] != 0ULL;
                    acc.w[q] = 0ULL;
                }
                if (any_need) {
                    // every lane ORs its neighbours' frontier words; the warp
                    // combines them (and tests for early exit) every 4 chunks
                    // of 32 neighbours -- extra ORs only add bits of the
                    // frontier, so the result does not depend on when it stops
                    const int32_t s = p.R[v], e = p.R[v + 1];
                    for (int32_t base = s; base < e; base += 128) {
#pragma unroll
                        for (int c = 0; c < 4; c++) {
                            const int32_t f = base + c * 32 + lane;
                            if (f < e) {
                                const Words<NW> fu = cur[p.C[f]];
#pragma unroll
                                for (int q = 0; q < NW; q++) acc.w[q] |= fu.w[q];
                            }
                        }
                        bool done = true;
#pragma unroll
                        for (int q = 0; q < NW; q++) {
                            const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)acc.w[q]);
                            const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(acc.w[q] >> 32));
                            acc.w[q] = ((unsigned long long)hi << 32) | lo;
                            done &= (acc.w[q] & need.w[q]) == need.w[q];
                        }
                        if (done) break;
                    }
                }
                int cnt = 0;
                Words<NW> nx, so;
#pragma unroll
                for (int q = 0; q < NW; q++) {
                    nx.w[q] = acc.w[q] & need.w[q];
                    so.w[q] = sv.w[q] | nx.w[q];
                    cnt += __popcll(nx.w[q]);
                }
                if (lane == 0) {
                    nxt[v] = nx;
                    sout[v] = so;
                    if (cnt) {
                        if (d <= MAX_D) p.cnt[(long long)v * MAX_D + (d - 1)] += (unsigned)cnt;
                        else p.inv_far[v] += (double)cnt / (double)d;
                    }
                }
                found_total += (unsigned)cnt;
            }
            if (lane == 0 && found_total && p.hist && d <= p.max_hop) atomicAdd(&p.hist[d], found_total);
            if (__syncthreads_or(found_total != 0) && threadIdx.x == 0) p.flags[d % 3] = 1;
            grid.sync();
            if (tid == 0) p.flags[(d + 2) % 3] = 0;   // last read before this barrier, next written after the next
            if (!((volatile int*)p.flags)[d % 3]) break;
            diam = max(diam, d);
            Words<NW>* t = sin; sin = sout; sout = t;
            t = cur; cur = nxt; nxt = t;
        }
    }
    if (tid == 0) *p.diameter = diam;
}

// inv[v] = sum_d cnt[v][d] / d (d ascending), eff[v] = inv[v] / (n - 1)
__global__ void k_inv_eff(PathArgs p)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < p.n; v += gridDim.x * blockDim.x) {
        double acc = 0.0;
        const unsigned* c = p.cnt + (long long)v * MAX_D;
        for (int d = 1; d <= MAX_D; d++)
            if (c[d - 1]) acc += (double)c[d - 1] / (double)d;
        acc += p.inv_far[v];
        p.inv[v] = acc;
        if (p.eff) p.eff[v] = p.n > 1 ? (float)(acc / (double)(p.n - 1)) : 0.0f;
    }
}

// total = sum_v inv[v] in a fixed order; lp = n(n-1)/total (0 without paths)
__global__ void k_lp(PathArgs p)
{
    __shared__ double sh[1024];
    const int n = p.n;
    double a = 0.0;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(n, lo + per);
    for (int i = lo; i < hi; i++) a += p.inv[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)blockDim.x; i++) t += sh[i];
        p.out[0] = t;
        p.out[1] = t > 0.0 ? (double)n * (double)(n - 1) / t : 0.0;
    }
}

template <int NW>
pg_status launch_all(pg_ctx* ctx, PathArgs& a, int ctas_per_sm)
{
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeCooperative;
    attr.val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctx->sm_count * ctas_per_sm);
    cfg.blockDim = dim3(THREADS);
    cfg.stream = ctx->stream;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_msbfs_all<NW>, a));
    PG_LAUNCHED(ctx);
    return PG_OK;
}

int max_ctas(pg_ctx* ctx, int nw)
{
    int per_sm = 0;
    cudaError_t e = nw == 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_msbfs_all<8>, THREADS, 0)
                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_msbfs_all<4>, THREADS, 0);
    (void)ctx;
    return e == cudaSuccess ? per_sm : 0;
}
}  // namespace

pg_status paths_prepare(pg_ctx* ctx, const pg_graph* g, int max_hop, PathArgs* a)
{
    const int n = g->n;
    memset(a, 0, sizeof *a);
    a->n = n;
    a->R = g->R;
    a->C = g->C;
    a->max_hop = max_hop;
    // both word widths share the buffers: sized for the wider one
    PG_TRY(pg_ws(ctx, "bfs.front", ((size_t)n + 1) * 64, &a->front));
    PG_TRY(pg_ws(ctx, "bfs.next", ((size_t)n + 1) * 64, &a->next));
    PG_TRY(pg_ws(ctx, "bfs.seen_a", ((size_t)n + 1) * 64, &a->seen_a));
    PG_TRY(pg_ws(ctx, "bfs.seen_b", ((size_t)n + 1) * 64, &a->seen_b));
    PG_TRY(pg_wst(ctx, "bfs.cnt", ((size_t)n + 1) * MAX_D, &a->cnt));
    PG_TRY(pg_wst(ctx, "bfs.inv_far", (size_t)n + 1, &a->inv_far));
    PG_TRY(pg_wst(ctx, "bfs.inv", (size_t)n + 1, &a->inv));
    PG_TRY(pg_wst(ctx, "bfs.eff", (size_t)n + 1, &a->eff));
    PG_TRY(pg_wst(ctx, "bfs.hist", (size_t)max_hop + 2, &a->hist));
    PG_TRY(pg_wst(ctx, "bfs.flags", 4, &a->flags));
    PG_TRY(pg_wst(ctx, "bfs.diam", 1, &a->diameter));
    PG_TRY(pg_wst(ctx, "bfs.out", 2, &a->out));
    // launch shape: sources per batch x CTAs per SM, from the autotuner
    const int cap4 = max_ctas(ctx, 4), cap8 = max_ctas(ctx, 8);
    if (cap4 < 1 || cap8 < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "paths: kernel does not fit an SM");
    std::vector<TuneChoice> cands;
    for (int nw : {4, 8})
        for (int c : {2, 4, 8})
            if (c <= (nw == 8 ? cap8 : cap4)) cands.push_back({nw, c});
    const std::string key = tune_key("msbfs", n, g->nnz);
    TuneChoice best{4, std::min(4, cap4)};
    PG_TRY(tune_pick(ctx, key, cands, &best, [&](const TuneChoice& c) -> pg_status {
        a->nw = c.a;
        a->ctas_per_sm = c.b;
        return paths_enqueue(ctx, a);
    }));
    a->nw = best.a;
    a->ctas_per_sm = best.b;
    return PG_OK;
}

pg_status paths_enqueue(pg_ctx* ctx, PathArgs* a)
{
    const int n = a->n;
    PG_CUDA(ctx, cudaMemsetAsync(a->cnt, 0, sizeof(unsigned) * ((size_t)n + 1) * MAX_D, ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(a->inv_far, 0, sizeof(double) * ((size_t)n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(a->hist, 0, sizeof(unsigned long long) * ((size_t)a->max_hop + 2), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(a->diameter, 0, sizeof(int), ctx->stream));
    if (n > 0) {
        if (a->nw == 8) PG_TRY(launch_all<8>(ctx, *a, a->ctas_per_sm));
        else PG_TRY(launch_all<4>(ctx, *a, a->ctas_per_sm));
    }
    const int grid = std::max(1, std::min(ctx->sm_count * 8, ceil_div(n, 256)));
    k_inv_eff<<<grid, 256, 0, ctx->stream>>>(*a);
    PG_LAUNCHED(ctx);
    k_lp<<<1, 1024, 0, ctx->stream>>>(*a);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

extern "C" pg_status pg_paths(pg_ctx* ctx, const pg_graph* g, float* eff, double* inv_sum, double* lp,
                              int64_t* hop_hist, int32_t max_hop, int32_t* diameter)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_paths: null argument");
    if (max_hop < 0) max_hop = 0;
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    PathArgs a;
    PG_TRY(paths_prepare(ctx, g, max_hop, &a));
    PG_TRY(paths_enqueue(ctx, &a));
    const int n = g->n;
    double out[2];
    PG_TRY(pg_d2h(ctx, out, a.out, sizeof out));
    if (eff) PG_TRY(pg_d2h(ctx, eff, a.eff, sizeof(float) * n));
    if (inv_sum) PG_TRY(pg_d2h(ctx, inv_sum, a.inv, sizeof(double) * n));
    if (hop_hist) {
        std::vector<unsigned long long> h(max_hop + 1);
        PG_TRY(pg_d2h(ctx, h.data(), a.hist, sizeof(unsigned long long) * (max_hop + 1)));
        for (int d = 0; d <= max_hop; d++) hop_hist[d] = (int64_t)h[d];
    }
    if (lp) *lp = out[1];
    if (diameter) {
        int dm = 0;
        PG_TRY(pg_d2h(ctx, &dm, a.diameter, sizeof dm));
        *diameter = dm;
    }
    return PG_OK;
}
