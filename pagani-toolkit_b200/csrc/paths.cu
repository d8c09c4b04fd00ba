// paths.cu -- hop path length and nodal efficiency (APSP_BFS,
// U/BFS_MulCPU/BFS_MulCPU/APSP_BFS.cpp:27-147) by bit-parallel multi-source
// BFS: 64*NW sources run together, one bit per source in NW 64-bit words per
// node.  A level is a pull sweep: node v ORs the frontier words of its
// neighbours, keeps the bits it has not seen, and stops scanning once every
// missing source bit is found.  Because the graph is undirected,
// d(s, v) = d(v, s): node v accumulates sum_s 1/d(s, v) directly, so the
// per-node efficiency needs no transposition or atomics.
#include "pg_internal.cuh"
#include <algorithm>

namespace {
constexpr int NW = 4;               // 256 sources per batch
constexpr int SRC_PER_BATCH = 64 * NW;

struct Words { unsigned long long w[NW]; };

__global__ void k_msbfs_init(int32_t n, int s0, int ns, Words* __restrict__ front, Words* __restrict__ seen)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        Words f;
#pragma unroll
        for (int q = 0; q < NW; q++) f.w[q] = 0ULL;
        int b = v - s0;
        if (b >= 0 && b < ns) f.w[b >> 6] = 1ULL << (b & 63);
        front[v] = f;
        seen[v] = f;
    }
}

// One level: warp per node.  Writes the next frontier, merges it into `seen`
// after the sweep (double buffered: seen_in -> seen_out), accumulates
// popcount/d into inv[v] and the hop histogram.
__global__ void k_msbfs_level(const int32_t* __restrict__ R, const int32_t* __restrict__ C, int32_t n,
                              const Words* __restrict__ front, Words* __restrict__ next,
                              const Words* __restrict__ seen_in, Words* __restrict__ seen_out, int d,
                              Words full, double* __restrict__ inv, unsigned long long* __restrict__ hist,
                              int max_hop, int* __restrict__ active)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long found_total = 0;
    for (int v = gw; v < n; v += nw) {
        Words sv = seen_in[v];
        Words need;
        bool any_need = false;
#pragma unroll
        for (int q = 0; q < NW; q++) { need.w[q] = full.w[q] & ~sv.w[q]; any_need |= need.w[q] != 0ULL; }
        Words acc;
#pragma unroll
        for (int q = 0; q < NW; q++) acc.w[q] = 0ULL;
        if (any_need) {
            const int32_t s = R[v], e = R[v + 1];
            for (int32_t base = s; base < e; base += 32) {
                int32_t f = base + lane;
                if (f < e) {
                    Words fu = front[C[f]];
#pragma unroll
                    for (int q = 0; q < NW; q++) acc.w[q] |= fu.w[q];
                }
                bool done = true;
#pragma unroll
                for (int q = 0; q < NW; q++) {
                    unsigned long long x = acc.w[q];
                    for (int o = 16; o; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
                    acc.w[q] = x;
                    done &= (x & need.w[q]) == need.w[q];
                }
                if (done) break;
            }
        }
        Words nx;
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < NW; q++) {
            nx.w[q] = acc.w[q] & need.w[q];
            cnt += __popcll(nx.w[q]);
        }
        if (lane == 0) {
            next[v] = nx;
            Words so;
#pragma unroll
            for (int q = 0; q < NW; q++) so.w[q] = sv.w[q] | nx.w[q];
            seen_out[v] = so;
            if (cnt) inv[v] += (double)cnt / (double)d;
        }
        found_total += cnt;
    }
    if (lane == 0 && found_total) {
        *active = 1;
        if (d <= max_hop) atomicAdd(&hist[d], found_total);
    }
}

__global__ void k_eff(const double* __restrict__ inv, int32_t n, float* __restrict__ eff)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        eff[v] = n > 1 ? (float)(inv[v] / (double)(n - 1)) : 0.0f;
}

__global__ void k_sum_f64(const double* __restrict__ x, int32_t n, double* __restrict__ out)
{
    __shared__ double sh[1024];
    double a = 0.0;
    int per = (n + blockDim.x - 1) / blockDim.x;
    int lo = threadIdx.x * per, hi = min(n, lo + per);
    for (int i = lo; i < hi; i++) a += x[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)blockDim.x; i++) t += sh[i];
        *out = t;
    }
}
}  // namespace

extern "C" pg_status pg_paths(pg_ctx* ctx, const pg_graph* g, float* eff, double* inv_sum, double* lp,
                              int64_t* hop_hist, int32_t max_hop, int32_t* diameter)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_paths: null argument");
    if (max_hop < 0) max_hop = 0;
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    Words *front, *next, *seen_a, *seen_b;
    double *inv, *tot;
    unsigned long long* hist;
    int* active;
    PG_TRY(pg_wst(ctx, "bfs.front", (size_t)n + 1, &front));
    PG_TRY(pg_wst(ctx, "bfs.next", (size_t)n + 1, &next));
    PG_TRY(pg_wst(ctx, "bfs.seen_a", (size_t)n + 1, &seen_a));
    PG_TRY(pg_wst(ctx, "bfs.seen_b", (size_t)n + 1, &seen_b));
    PG_TRY(pg_wst(ctx, "bfs.inv", (size_t)n + 1, &inv));
    PG_TRY(pg_wst(ctx, "bfs.tot", 1, &tot));
    PG_TRY(pg_wst(ctx, "bfs.hist", (size_t)max_hop + 2, &hist));
    PG_TRY(pg_wst(ctx, "bfs.active", 64, &active));
    PG_CUDA(ctx, cudaMemsetAsync(inv, 0, sizeof(double) * (n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * (max_hop + 2), ctx->stream));
    int* hact;
    PG_TRY(pg_pinned(ctx, 4096, (void**)&hact));
    int diam = 0;
    const int grid_nodes = std::max(1, std::min(ctx->sm_count * 16, ceil_div(n, 256)));
    const int grid_warps = std::max(1, std::min(ctx->sm_count * 16, ceil_div((long long)n * 32, 256)));
    for (int s0 = 0; s0 < n; s0 += SRC_PER_BATCH) {
        const int ns = std::min(SRC_PER_BATCH, n - s0);
        Words full;
        for (int q = 0; q < NW; q++) {
            int lo = q * 64, c = std::max(0, std::min(64, ns - lo));
            full.w[q] = c == 64 ? ~0ULL : (c ? ((1ULL << c) - 1ULL) : 0ULL);
        }
        k_msbfs_init<<<grid_nodes, 256, 0, ctx->stream>>>(n, s0, ns, front, seen_a);
        PG_LAUNCHED(ctx);
        Words *sin = seen_a, *sout = seen_b, *cur = front, *nxt = next;
        for (int d = 1; d <= n; d++) {
            PG_CUDA(ctx, cudaMemsetAsync(active, 0, sizeof(int), ctx->stream));
            k_msbfs_level<<<grid_warps, 256, 0, ctx->stream>>>(g->R, g->C, n, cur, nxt, sin, sout, d, full, inv,
                                                               hist, max_hop, active);
            PG_LAUNCHED(ctx);
            PG_CUDA(ctx, cudaMemcpyAsync(hact, active, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (!*hact) break;
            diam = std::max(diam, d);
            std::swap(sin, sout);
            std::swap(cur, nxt);
        }
    }
    float* deff;
    PG_TRY(pg_wst(ctx, "bfs.eff", (size_t)n + 1, &deff));
    k_eff<<<grid_nodes, 256, 0, ctx->stream>>>(inv, n, deff);
    PG_LAUNCHED(ctx);
    k_sum_f64<<<1, 1024, 0, ctx->stream>>>(inv, n, tot);
    PG_LAUNCHED(ctx);
    double total = 0.0;
    PG_TRY(pg_d2h(ctx, &total, tot, sizeof(double)));
    if (eff) PG_TRY(pg_d2h(ctx, eff, deff, sizeof(float) * n));
    if (inv_sum) PG_TRY(pg_d2h(ctx, inv_sum, inv, sizeof(double) * n));
    if (hop_hist) {
        std::vector<unsigned long long> h(max_hop + 1);
        PG_TRY(pg_d2h(ctx, h.data(), hist, sizeof(unsigned long long) * (max_hop + 1)));
        for (int d = 0; d <= max_hop; d++) hop_hist[d] = (int64_t)h[d];
    }
    if (lp) *lp = total > 0.0 ? (double)n * (double)(n - 1) / total : 0.0;
    if (diameter) *diameter = diam;
    return PG_OK;
}
