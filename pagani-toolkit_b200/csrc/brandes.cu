// brandes.cu -- Brandes betweenness from all sources (CUBC, U/BC/CUBC/
// BC_GPU_node_pred.cu:6-155; Betweenness_CPU, U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:6-82)
// with exact 64-bit path counts and FP64 dependencies.
//
// 128 sources run together, four per warp lane (lane l owns sources l,
// l+32, l+64, l+96): per node the state is a row of 128 entries (level int32,
// sigma uint64, coefficient double), so a neighbour's state for all sources
// is four coalesced 256-byte reads.  Source bits are 128-bit masks per node
// (two 64-bit words).
//   forward level d:  node v sums sigma[u][s] over neighbours u that are in
//                     the frontier of a source s not yet seen at v; the
//                     non-zero sums are exactly the sources reaching v at d;
//   backward level d: v on level d of source s sums
//                     (1 + delta[w][s]) / sigma[w][s] over neighbours w on
//                     level d+1 (stored as one coefficient per entry), so
//                     delta[v][s] = sigma[v][s] * sum; BC[v] += sum_s delta.
// Neighbours are visited 32 at a time; a ballot over the 32 frontier masks
// keeps only those that matter for some source, and those are broadcast to
// the warp one by one.  The frontier mask of every level (< LCAP) is kept so
// the backward sweep filters neighbours the same way.
// BC[v] is the sum over ORDERED (source, target) pairs like the reference.
// The whole sweep is a cooperative kernel; levels are separated by grid-wide
// barriers (no host round trip per level).  The forward pass also yields the
// hop path length (sum of 1/d per node), returned by pg_betweenness on request.
#include "pg_internal.cuh"
#include "bc_dense.cuh"
#include <cooperative_groups.h>
#include <climits>
#include <algorithm>

namespace cg = cooperative_groups;

namespace {
constexpr int THREADS = 256;
constexpr int S = 128;        // sources per batch
constexpr int SL = S / 32;    // sources per lane
constexpr int LCAP = 48;      // levels whose frontier masks are kept for the backward sweep
typedef unsigned long long u64;

struct BCArgs {
    const int32_t* R;
    const int32_t* C;
    int32_t n;
    const int32_t* sources;   // null: sources 0..n-1
    int32_t nsrc;
    int32_t* dist;            // [n][S]
    u64* sigma;               // [n][S]
    double* coef;             // [n][S]
    ulonglong2* front;        // [2][n] source masks (x: sources 0-63, y: 64-127)
    ulonglong2* fhist;        // [LCAP][n] frontier mask of every level < LCAP
    ulonglong2* seen;         // [n]
    int* flags;               // [3] rotating "something changed" flags
    double* bc;               // [n] accumulated FP64 betweenness (null: forward only)
    double* inv;              // [n] sum of 1/d (null: skip)
    int do_backward;
    int32_t* out_dist;        // pg_bfs_sigma output of one batch (null otherwise)
    u64* out_sigma;
    const int32_t* order;     // nodes by decreasing degree (largest work first)
    int* work;                // [WORK_SLOTS] per-level work counters
};

constexpr int WORK_SLOTS = 4096;   // forward + backward levels per batch with dynamic scheduling

// Next node for this warp: nodes are handed out in order of decreasing
// degree through one atomic counter per level, so hubs start first and no
// warp idles at the level barrier while another still holds a long list.
// Levels beyond the counter array fall back to a static interleave.
__device__ __forceinline__ int next_node(const BCArgs& a, int slot, int& k, int gw, int nw)
{
    if (slot >= WORK_SLOTS) {
        int v = gw + k * nw;
        k++;
        return v < a.n ? v : a.n;
    }
    int idx = 0;
    if ((threadIdx.x & 31) == 0) idx = atomicAdd(&a.work[slot], 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    return idx < a.n ? a.order[idx] : a.n;
}

__device__ __forceinline__ u64 shfl64(u64 x, int j) { return __shfl_sync(0xffffffffu, x, j); }

// bit of source lane + 32 k in a 128-bit mask
__device__ __forceinline__ bool has_src(const ulonglong2& m, int lane, int k)
{
    const u64 w = k < 2 ? m.x : m.y;
    return (w >> (lane + 32 * (k & 1))) & 1ULL;
}

// Per 32-neighbour chunk the sweeps pick one of two layouts:
//  - by neighbour: the warp takes the active neighbours one by one and every
//    lane handles its four sources (all 128 sources per neighbour step);
//  - by source: lanes hold the 32 neighbours and the warp walks the sources
//    the node still needs, one warp-wide sum per source.
// The cost of a chunk is about BY_NB per active neighbour in the first and
// BY_SRC_* per needed source in the second (tuned on the 58k subject graphs);
// the cheaper one runs.  Late forward levels and the first backward level
// need few sources per node.
constexpr int BY_NB = 40, BY_SRC_FWD = 96, BY_SRC_BWD = 32;

__device__ __forceinline__ int next_src(u64& w0, u64& w1)
{
    if (w0) {
        const int s = __ffsll((long long)w0) - 1;
        w0 &= w0 - 1;
        return s;
    }
    if (w1) {
        const int s = 64 + __ffsll((long long)w1) - 1;
        w1 &= w1 - 1;
        return s;
    }
    return -1;
}

__device__ __forceinline__ bool mask_bit(const ulonglong2& m, int s)
{
    return ((s < 64 ? m.x : m.y) >> (s & 63)) & 1ULL;
}

// mask with bit lane + 32 k set where f[k] holds, over the warp
__device__ __forceinline__ ulonglong2 lane_mask(const bool (&f)[SL])
{
    const unsigned b0 = __ballot_sync(0xffffffffu, f[0]), b1 = __ballot_sync(0xffffffffu, f[1]);
    const unsigned b2 = __ballot_sync(0xffffffffu, f[2]), b3 = __ballot_sync(0xffffffffu, f[3]);
    return make_ulonglong2((u64)b0 | ((u64)b1 << 32), (u64)b2 | ((u64)b3 << 32));
}

// four CTAs per SM (64 registers): occupancy hides the L2 latency of the row gathers
// Batches [batch_first, batch_last); the forward sweep runs levels
// fwd_first..fwd_last.  fwd_first > 1 resumes a batch whose earlier levels
// were computed elsewhere (the dense tensor-core levels); fwd_last < INT_MAX
// stops after that level, before the backward sweep (one batch per launch).
__global__ void __launch_bounds__(THREADS, 4)
k_brandes(BCArgs a, int batch_first, int batch_last, int fwd_first, int fwd_last)
{
    cg::grid_group grid = cg::this_grid();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int n = a.n;
    const size_t gt = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
    for (int b = batch_first; b < batch_last; b++) {
        const int s0 = b * S;
        const int ns = min(S, a.nsrc - s0);
        const ulonglong2 full = make_ulonglong2(ns >= 64 ? ~0ULL : ((1ULL << ns) - 1ULL),
                                                ns >= 128 ? ~0ULL : ns > 64 ? ((1ULL << (ns - 64)) - 1ULL) : 0ULL);
        const bool init = fwd_first <= 1;
        // ---- init: levels -1, frontier = sources
        for (size_t q = gt; init && q < (size_t)n * S; q += gstride) a.dist[q] = -1;
        for (size_t v = gt; init && v < (size_t)n; v += gstride) {
            a.front[v] = make_ulonglong2(0ULL, 0ULL);
            a.seen[v] = make_ulonglong2(0ULL, 0ULL);
            a.fhist[v] = make_ulonglong2(0ULL, 0ULL);
        }
        for (size_t q = gt; init && q < (size_t)WORK_SLOTS; q += gstride) a.work[q] = 0;
        if (init && gt < 3) a.flags[gt] = 0;
        grid.sync();
        if (init && gt < (size_t)ns) {
            int s = a.sources ? a.sources[s0 + gt] : s0 + (int)gt;
            a.dist[(size_t)s * S + gt] = 0;
            a.sigma[(size_t)s * S + gt] = 1ULL;
            const u64 bit = 1ULL << (gt & 63);
            u64* w = gt < 64 ? &a.front[s].x : &a.front[s].y;
            atomicOr(w, bit);
            atomicOr(gt < 64 ? &a.seen[s].x : &a.seen[s].y, bit);
            atomicOr(gt < 64 ? &a.fhist[s].x : &a.fhist[s].y, bit);
        }
        grid.sync();
        // ---- forward: level d reads the frontier buffer (d - 1) & 1 and writes d & 1
        int d = init ? 1 : fwd_first;
        ulonglong2* cur = a.front + (size_t)((d - 1) & 1) * n;
        ulonglong2* nxt = a.front + (size_t)(d & 1) * n;
        if (!init) {
            if (gt == 0) a.flags[d % 3] = 0;
            grid.sync();
        }
        bool stopped = false;
        for (;; d++) {
            if (gt == 0) a.flags[(d + 1) % 3] = 0;
            int found = 0;
            int kk = 0;
            const int fslot = d < WORK_SLOTS / 2 ? d : WORK_SLOTS;
            for (int v = next_node(a, fslot, kk, gw, nw); v < n; v = next_node(a, fslot, kk, gw, nw)) {
                const ulonglong2 sv = a.seen[v];
                const ulonglong2 need = make_ulonglong2(full.x & ~sv.x, full.y & ~sv.y);
                ulonglong2 nb = make_ulonglong2(0ULL, 0ULL);
                if (need.x | need.y) {
                    const int32_t s = a.R[v], e = a.R[v + 1];
                    const int kneed = __popcll(need.x) + __popcll(need.y);
                    u64 sg[SL] = {0ULL, 0ULL, 0ULL, 0ULL};
                    for (int32_t base = s; base < e; base += 32) {
                        int32_t f = base + lane;
                        int u = f < e ? a.C[f] : 0;
                        ulonglong2 fu = make_ulonglong2(0ULL, 0ULL);
                        if (f < e) {
                            const ulonglong2 c = cur[u];
                            fu = make_ulonglong2(c.x & need.x, c.y & need.y);
                        }
                        unsigned m = __ballot_sync(0xffffffffu, (fu.x | fu.y) != 0ULL);
                        if (m && kneed * BY_SRC_FWD < __popc(m) * BY_NB) {
                            // by source, two at a time; integer sums, exact in any order
                            u64 w0 = need.x, w1 = need.y;
                            for (;;) {
                                const int sa = next_src(w0, w1), sb = next_src(w0, w1);
                                if (sa < 0) break;
                                u64 xa = mask_bit(fu, sa) ? a.sigma[(size_t)u * S + sa] : 0ULL;
                                u64 xb = (sb >= 0 && mask_bit(fu, sb)) ? a.sigma[(size_t)u * S + sb] : 0ULL;
#pragma unroll
                                for (int o = 16; o; o >>= 1) {
                                    xa += __shfl_xor_sync(0xffffffffu, xa, o);
                                    xb += __shfl_xor_sync(0xffffffffu, xb, o);
                                }
                                {
                                    const u64 adda = lane == (sa & 31) ? xa : 0ULL;
                                    const u64 addb = (sb >= 0 && lane == (sb & 31)) ? xb : 0ULL;
                                    const int ka = sa >> 5, kb = sb >> 5;
                                    sg[0] += (ka == 0 ? adda : 0ULL) + (kb == 0 ? addb : 0ULL);
                                    sg[1] += (ka == 1 ? adda : 0ULL) + (kb == 1 ? addb : 0ULL);
                                    sg[2] += (ka == 2 ? adda : 0ULL) + (kb == 2 ? addb : 0ULL);
                                    sg[3] += (ka == 3 ? adda : 0ULL) + (kb == 3 ? addb : 0ULL);
                                }
                            }
                            m = 0u;
                        }
                        // by neighbour: two active neighbours per step, their loads issued together
                        while (m) {
                            int j[2];
#pragma unroll
                            for (int t = 0; t < 2; t++) {
                                j[t] = m ? __ffs(m) - 1 : -1;
                                m &= m ? m - 1 : 0u;
                            }
                            u64 x[2][SL];
#pragma unroll
                            for (int t = 0; t < 2; t++) {
                                const int jj = j[t] < 0 ? j[0] : j[t];
                                const int uj = __shfl_sync(0xffffffffu, u, jj);
                                ulonglong2 fj;
                                fj.x = j[t] < 0 ? 0ULL : shfl64(fu.x, jj);
                                fj.y = j[t] < 0 ? 0ULL : shfl64(fu.y, jj);
                                const u64* row = a.sigma + (size_t)uj * S;
#pragma unroll
                                for (int k = 0; k < SL; k++) x[t][k] = has_src(fj, lane, k) ? row[lane + 32 * k] : 0ULL;
                            }
#pragma unroll
                            for (int t = 0; t < 2; t++)
#pragma unroll
                                for (int k = 0; k < SL; k++) sg[k] += x[t][k];
                        }
                    }
                    const bool fs[SL] = {sg[0] != 0ULL, sg[1] != 0ULL, sg[2] != 0ULL, sg[3] != 0ULL};
                    nb = lane_mask(fs);
#pragma unroll
                    for (int k = 0; k < SL; k++)
                        if (sg[k]) {
                            a.sigma[(size_t)v * S + lane + 32 * k] = sg[k];
                            a.dist[(size_t)v * S + lane + 32 * k] = d;
                        }
                    if (nb.x | nb.y) {
                        if (lane == 0 && a.inv) a.inv[v] += (double)(__popcll(nb.x) + __popcll(nb.y)) / (double)d;
                        found = 1;
                    }
                }
                if (lane == 0) {
                    nxt[v] = nb;
                    a.seen[v] = make_ulonglong2(sv.x | nb.x, sv.y | nb.y);
                    if (d < LCAP) a.fhist[(size_t)d * n + v] = nb;
                }
            }
            if (found && lane == 0) a.flags[d % 3] = 1;
            grid.sync();
            const int any = a.flags[d % 3];
            ulonglong2* t = cur; cur = nxt; nxt = t;
            if (d >= fwd_last) {
                stopped = true;
                break;
            }
            if (!any) break;
        }
        if (stopped) continue;   // the caller computes the next levels
        const int maxd = d - 1;  // deepest level reached
        if (a.out_dist) {
            for (size_t q = gt; q < (size_t)ns * n; q += gstride) {
                size_t sidx = q / n, v = q % n;
                a.out_dist[q] = a.dist[v * S + sidx];
                a.out_sigma[q] = a.dist[v * S + sidx] >= 0 ? a.sigma[v * S + sidx] : 0ULL;
            }
        }
        // ---- backward
        if (a.do_backward) {
            for (int lv = maxd; lv >= 1; lv--) {
                // backward levels use the upper half of the counters
                const int bslot = lv < WORK_SLOTS / 2 ? WORK_SLOTS / 2 + lv : WORK_SLOTS;
                int kk = 0;
                for (int v = next_node(a, bslot, kk, gw, nw); v < n; v = next_node(a, bslot, kk, gw, nw)) {
                    // sources for which v sits on level lv
                    ulonglong2 mine;
                    if (lv < LCAP) {
                        mine = a.fhist[(size_t)lv * n + v];
                    } else {
                        bool on[SL];
#pragma unroll
                        for (int k = 0; k < SL; k++) on[k] = a.dist[(size_t)v * S + lane + 32 * k] == lv;
                        mine = lane_mask(on);
                    }
                    if (!(mine.x | mine.y)) continue;
                    double acc[SL] = {0.0, 0.0, 0.0, 0.0};
                    if (lv < maxd) {
                        const int32_t s = a.R[v], e = a.R[v + 1];
                        const int kmine = __popcll(mine.x) + __popcll(mine.y);
                        for (int32_t base = s; base < e; base += 32) {
                            int32_t f = base + lane;
                            int w = f < e ? a.C[f] : 0;
                            if (lv + 1 < LCAP) {
                                // neighbours one level deeper for some of v's sources
                                ulonglong2 mw = make_ulonglong2(0ULL, 0ULL);
                                if (f < e) {
                                    const ulonglong2 h = a.fhist[(size_t)(lv + 1) * n + w];
                                    mw = make_ulonglong2(h.x & mine.x, h.y & mine.y);
                                }
                                unsigned bm = __ballot_sync(0xffffffffu, (mw.x | mw.y) != 0ULL);
                                if (bm && kmine * BY_SRC_BWD < __popc(bm) * BY_NB) {
                                    // by source, two at a time; each chunk's terms meet in a
                                    // fixed shuffle tree, so the FP64 sums are deterministic
                                    u64 w0 = mine.x, w1 = mine.y;
                                    for (;;) {
                                        const int sa = next_src(w0, w1), sb = next_src(w0, w1);
                                        if (sa < 0) break;
                                        double xa = mask_bit(mw, sa) ? a.coef[(size_t)w * S + sa] : 0.0;
                                        double xb = (sb >= 0 && mask_bit(mw, sb)) ? a.coef[(size_t)w * S + sb] : 0.0;
#pragma unroll
                                        for (int o = 16; o; o >>= 1) {
                                            xa += __shfl_xor_sync(0xffffffffu, xa, o);
                                            xb += __shfl_xor_sync(0xffffffffu, xb, o);
                                        }
                                        {
                                            const double adda = lane == (sa & 31) ? xa : 0.0;
                                            const double addb = (sb >= 0 && lane == (sb & 31)) ? xb : 0.0;
                                            const int ka = sa >> 5, kb = sb >> 5;
                                            if (ka == 0) acc[0] += adda;
                                            if (ka == 1) acc[1] += adda;
                                            if (ka == 2) acc[2] += adda;
                                            if (ka == 3) acc[3] += adda;
                                            if (kb == 0) acc[0] += addb;
                                            if (kb == 1) acc[1] += addb;
                                            if (kb == 2) acc[2] += addb;
                                            if (kb == 3) acc[3] += addb;
                                        }
                                    }
                                    bm = 0u;
                                }
                                while (bm) {
                                    int j[2];
#pragma unroll
                                    for (int t = 0; t < 2; t++) {
                                        j[t] = bm ? __ffs(bm) - 1 : -1;
                                        bm &= bm ? bm - 1 : 0u;
                                    }
                                    double y[2][SL];
#pragma unroll
                                    for (int t = 0; t < 2; t++) {
                                        const int jj = j[t] < 0 ? j[0] : j[t];
                                        const int wj = __shfl_sync(0xffffffffu, w, jj);
                                        ulonglong2 mj;
                                        mj.x = j[t] < 0 ? 0ULL : shfl64(mw.x, jj);
                                        mj.y = j[t] < 0 ? 0ULL : shfl64(mw.y, jj);
                                        const double* row = a.coef + (size_t)wj * S;
#pragma unroll
                                        for (int k = 0; k < SL; k++) y[t][k] = has_src(mj, lane, k) ? row[lane + 32 * k] : 0.0;
                                    }
#pragma unroll
                                    for (int t = 0; t < 2; t++)
#pragma unroll
                                        for (int k = 0; k < SL; k++) acc[k] += y[t][k];
                                }
                            } else {
                                int cnt = min(32, e - base);
                                for (int jn = 0; jn < cnt; jn++) {
                                    int wj = __shfl_sync(0xffffffffu, w, jn);
                                    const int32_t* dw = a.dist + (size_t)wj * S;
                                    const double* row = a.coef + (size_t)wj * S;
#pragma unroll
                                    for (int k = 0; k < SL; k++)
                                        if (has_src(mine, lane, k) && dw[lane + 32 * k] == lv + 1) acc[k] += row[lane + 32 * k];
                                }
                            }
                        }
                    }
                    double delta = 0.0;
#pragma unroll
                    for (int k = 0; k < SL; k++)
                        if (has_src(mine, lane, k)) {
                            const size_t at = (size_t)v * S + lane + 32 * k;
                            const double sg = __ull2double_rn(a.sigma[at]);
                            const double dl = sg * acc[k];
                            a.coef[at] = (1.0 + dl) / sg;
                            delta += dl;
                        }
                    for (int o = 16; o; o >>= 1) delta += __shfl_xor_sync(0xffffffffu, delta, o);
                    if (lane == 0 && a.bc) a.bc[v] += delta;
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

pg_status alloc_state(pg_ctx* ctx, int n, BCArgs& a, int* max_deg = nullptr)
{
    PG_TRY(pg_wst(ctx, "bc.dist", (size_t)n * S + S, &a.dist));
    PG_TRY(pg_wst(ctx, "bc.sigma", (size_t)n * S + S, &a.sigma));
    PG_TRY(pg_wst(ctx, "bc.coef", (size_t)n * S + S, &a.coef));
    PG_TRY(pg_wst(ctx, "bc.front", (size_t)2 * n + 2, &a.front));
    PG_TRY(pg_wst(ctx, "bc.fhist", (size_t)LCAP * n + 2, &a.fhist));
    PG_TRY(pg_wst(ctx, "bc.seen", (size_t)n + 1, &a.seen));
    PG_TRY(pg_wst(ctx, "bc.flags", 4, &a.flags));
    PG_TRY(pg_wst(ctx, "bc.work", (size_t)WORK_SLOTS, &a.work));
    // nodes by decreasing degree (stable), for the dynamic level schedule
    std::vector<int32_t> hR((size_t)n + 1), ord(n);
    PG_TRY(pg_d2h(ctx, hR.data(), a.R, sizeof(int32_t) * (n + 1)));
    for (int i = 0; i < n; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return hR[x + 1] - hR[x] > hR[y + 1] - hR[y]; });
    if (max_deg) *max_deg = n > 0 ? hR[ord[0] + 1] - hR[ord[0]] : 0;
    int32_t* dord;
    PG_TRY(pg_wst(ctx, "bc.order", (size_t)n + 1, &dord));
    PG_TRY(pg_h2d(ctx, dord, ord.data(), sizeof(int32_t) * n));
    a.order = dord;
    return PG_OK;
}

pg_status launch_brandes(pg_ctx* ctx, BCArgs& a, int batch_first, int batch_last, int fwd_first = 1,
                         int fwd_last = INT_MAX)
{
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_brandes, THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "brandes kernel cannot be resident");
    int grid = per_sm * ctx->sm_count;
    void* args[] = {(void*)&a, (void*)&batch_first, (void*)&batch_last, (void*)&fwd_first, (void*)&fwd_last};
    const int prof = pg_prof_begin(ctx, "k_brandes");
    PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_brandes, dim3(grid), dim3(THREADS), args, 0, ctx->stream));
    PG_LAUNCHED(ctx);
    pg_prof_end(ctx, prof);
    return PG_OK;
}

// Levels 2 and 3 of every batch on the tensor cores (dense graphs): level 1
// by the gather kernel, 2 and 3 as exact integer GEMMs, the rest (and the
// backward sweep) by the gather kernel again.
constexpr int DENSE_FIRST = 2, DENSE_LAST = 3;

pg_status dense_batch(pg_ctx* ctx, BCArgs& a, int b, BCDense& dn)
{
    PG_TRY(launch_brandes(ctx, a, b, b + 1, 1, DENSE_FIRST - 1));
    for (int d = DENSE_FIRST; d <= DENSE_LAST; d++) {
        BCLevel lv;
        lv.sigma = a.sigma;
        lv.dist = a.dist;
        lv.seen = a.seen;
        lv.nxt = a.front + (size_t)(d & 1) * a.n;
        lv.fprev = a.front + (size_t)((d - 1) & 1) * a.n;
        lv.fhist = d < LCAP ? a.fhist + (size_t)d * a.n : nullptr;
        lv.inv = a.inv;
        lv.flag = nullptr;
        lv.d = d;
        PG_TRY(bc_dense_level(ctx, dn, lv));
    }
    return launch_brandes(ctx, a, b, b + 1, DENSE_LAST + 1, INT_MAX);
}

pg_status run_batches(pg_ctx* ctx, BCArgs& a, int nb, BCDense* dn)
{
    if (!dn) {
        const int per_launch = 16;   // a bounded number of batches per launch keeps every launch short
        for (int b = 0; b < nb; b += per_launch) PG_TRY(launch_brandes(ctx, a, b, std::min(nb, b + per_launch)));
        return PG_OK;
    }
    for (int b = 0; b < nb; b++) PG_TRY(dense_batch(ctx, a, b, *dn));
    return bc_dense_check(ctx, *dn);
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
    BCDense dn;
    PG_TRY(alloc_state(ctx, n, a, &dn.max_deg));
    const bool dense = bc_dense_eligible(ctx, n, g->nnz, dn.max_deg);
    if (dense) PG_TRY(bc_dense_setup(ctx, g->R, g->C, n, dn));
    PG_TRY(pg_wst(ctx, "bc.bc", (size_t)n + 1, &a.bc));
    PG_CUDA(ctx, cudaMemsetAsync(a.bc, 0, sizeof(double) * (n + 1), ctx->stream));
    if (eff || lp) {
        PG_TRY(pg_wst(ctx, "bc.inv", (size_t)n + 1, &a.inv));
        PG_CUDA(ctx, cudaMemsetAsync(a.inv, 0, sizeof(double) * (n + 1), ctx->stream));
    }
    PG_TRY(run_batches(ctx, a, (n + S - 1) / S, dense ? &dn : nullptr));
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
    BCDense dn;
    PG_TRY(alloc_state(ctx, n, a, &dn.max_deg));
    const bool dense = bc_dense_eligible(ctx, n, g->nnz, dn.max_deg);
    if (dense) PG_TRY(bc_dense_setup(ctx, g->R, g->C, n, dn));
    int32_t* dsrc;
    PG_TRY(pg_wst(ctx, "bc.src", (size_t)ns + 1, &dsrc));
    PG_CUDA(ctx, cudaMemcpyAsync(dsrc, sources, sizeof(int32_t) * ns, cudaMemcpyHostToDevice, ctx->stream));
    a.sources = dsrc;
    PG_TRY(pg_wst(ctx, "bc.odist", (size_t)S * n, &a.out_dist));
    PG_TRY(pg_wst(ctx, "bc.osigma", (size_t)S * n, &a.out_sigma));
    for (int b = 0; b < (ns + S - 1) / S; b++) {
        if (dense) {
            PG_TRY(dense_batch(ctx, a, b, dn));
            PG_TRY(bc_dense_check(ctx, dn));
        } else {
            PG_TRY(launch_brandes(ctx, a, b, b + 1));
        }
        int cnt = std::min(S, ns - b * S);
        PG_TRY(pg_d2h(ctx, dist + (size_t)b * S * n, a.out_dist, sizeof(int32_t) * (size_t)cnt * n));
        PG_TRY(pg_d2h(ctx, sigma + (size_t)b * S * n, a.out_sigma, sizeof(int64_t) * (size_t)cnt * n));
    }
    return PG_OK;
}
