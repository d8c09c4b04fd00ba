// fw.cu -- weighted path length by blocked Floyd-Warshall in FP32 min-plus
// (CUBFW_Lp, W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp.cpp:13-162; phases of cuAPSP,
// CUBFW.cpp:19-168, CUBFW_ph1/2/3.cu, and BFW_C, BFW.cpp:40-109) and Onnela
// weighted clustering (Cp_2, W/Cp/Cp/Cp_2.cpp:23-130) for one graph or a
// batch of graphs in ONE persistent cooperative launch.
//
// Every graph's dense distance matrix (padded to a multiple of 64) stays in
// HBM for the whole sweep (the reference streams 3072^2 blocks over PCIe per
// phase and pads every graph to 3072).  The launch runs, with grid-wide
// barriers between them:
//   A  matrices set to +inf (0 on the diagonal); the weight maximum of every
//      graph (the Onnela normalisation);
//   B  edge distances 1/w and the cube roots of the normalised weights;
//      then Onnela clustering of every node of every graph (one CTA per
//      node, dynamic scheduler, the node's row dense in shared memory);
//   then for every 64-wide k-block round kb, over all graphs with more than
//   kb blocks at once (graphs are sorted by block count, so the active ones
//   are a prefix of the order):
//   1  closure of the diagonal block in shared memory, 64 steps, one barrier
//      per step (row and column k are fixed during step k: d_kk = 0);
//   2  the row and column panels against the closed diagonal block, in
//      place, likewise;
//   3  every other block: d_ij = min(d_ij, d_i,kb (x) d_kb,j) as a register-
//      tiled min-plus product -- 4 x 4 outputs per thread, the kb column
//      block transposed into shared memory so both operands are 16-byte
//      vector loads, no barrier inside the k loop (the reference's phase 3
//      keeps 6 x 6 per thread with scalar shared loads, CUBFW_ph3.cu:32-222);
//   C  per-row sums of 1/d (CUBFW_Lp.cpp:77-104), then per graph Lp and the
//      mean clustering.
// The k-block width is fixed (64), so the distances do not depend on any
// tuning; the autotuner only picks the CTAs per SM.
#include "pg_internal.cuh"
#include "tune.cuh"
#include <algorithm>
#include <cmath>
#include <cooperative_groups.h>
#include <numeric>

namespace cg = cooperative_groups;

namespace {
constexpr int B = 64;           // k-block width
constexpr int FW_THREADS = 256; // 16 x 16 threads, 4 x 4 outputs each
constexpr int ONNELA_MAX_N = 4096; // largest graph of a batch for the Onnela row (n doubles in shared memory)

struct FWGraph {
    const int32_t* R;
    const int32_t* C;
    const float* V;     // null: every edge has distance 1
    int32_t n, np, nb;  // nodes, padded size, blocks per side
    long long off;      // matrix offset (elements)
    int32_t node0;      // offset of its nodes in concatenated outputs
};

struct FwBatch {
    const FWGraph* gs;          // in processing order (blocks per side descending)
    int ng;
    int total_nodes;
    int max_nb;
    const int* active;          // [kb]: graphs with more than kb blocks (a prefix of gs)
    const long long* p2;        // prefix over gs of 2 (nb - 1): panel tasks
    const long long* p3;        // prefix over gs of (nb - 1)^2: phase-3 tasks
    const long long* edge0;     // offset of each graph's edges in cw
    const int* node_graph;      // concatenated node -> index in gs
    float* D;
    float* vmax;
    double* cw;                 // per edge of every graph: (V / vmax)^(1/3)
    int* onnela_next;           // dynamic node scheduler
    int onnela;                 // compute the clustering
    double* rowsum;             // per node
    float* eff;                 // per node
    double* lp;                 // per graph (in gs order)
    float* cp;                  // per node
    double* cp_mean;            // per graph (in gs order)
};

__device__ __forceinline__ float* blk(float* D, const FWGraph& g, int bi, int bj)
{
    return D + g.off + (long long)bi * B * g.np + (long long)bj * B;
}

// graph of task t in a prefix array of `count` graphs
__device__ __forceinline__ int task_graph(const long long* pre, int count, long long t)
{
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Onnela for node x of the batch (W/Cp/Cp/Cp_2.cpp:23-130, GPU weight maximum
// over all edges): sum over connected neighbour pairs j < h of
// (w_jh w_uj w_uh)^(1/3), w = V / vmax (float division), computed as
// cw_jh cw_uj cw_uh with the per-edge cube roots cw = w^(1/3) (FP64; the
// same value up to rounding).  u's row is spread into a dense shared-memory
// array (zero where h is not a neighbour), so the weight of (u, h) is one
// shared load.
__device__ void onnela_node(const FwBatch& p, int x, double* row, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = FW_THREADS / 32;
    const int gi = p.node_graph[x];
    const FWGraph g = p.gs[gi];
    const long long e0 = p.edge0[gi];
    const int u = x - g.node0;
    const int32_t s = g.R[u], e = g.R[u + 1];
    const int k = e - s;
    double acc = 0.0;
    if (k >= 2) {
        for (int32_t q = s + threadIdx.x; q < e; q += FW_THREADS) row[g.C[q]] = p.cw[e0 + q];
        __syncthreads();
        for (int32_t q = s + warp; q < e; q += nwarp) {
            const int j = g.C[q];
            const double cuj = p.cw[e0 + q];
            double part = 0.0;
            for (int32_t f = g.R[j] + lane; f < g.R[j + 1]; f += 32) {
                const int h = g.C[f];
                if (h > j) part += p.cw[e0 + f] * row[h];
            }
            acc += cuj * part;
        }
        __syncthreads();
        for (int32_t q = s + threadIdx.x; q < e; q += FW_THREADS) row[g.C[q]] = 0.0;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nwarp; w++) t += red[w];
        p.cp[x] = k >= 2 ? (float)(2.0 * t / k / (k - 1)) : 0.0f;
    }
    __syncthreads();
}

// Closure of a 64 x 64 block held in registers (4 x 4 per thread, rows
// 4 ty.., columns 4 tx..) against the diagonal block: mode 0 the diagonal
// block itself, 1 a row panel (s = min(s, dg (x) s)), 2 a column panel
// (s = min(s, s (x) dg)).  Row k and column k do not change in step k
// (d_kk = 0), so at every step their owners publish them to shared rows
// (double-buffered: one barrier per step) and every thread updates its tile
// from 16-byte loads; the closed diagonal block is read from dgT (its
// columns stored as rows) or dg.
__device__ __forceinline__ void closure(float (&acc)[4][4], const float (*dg)[B + 4], const float (*dgT)[B + 4],
                                        float (*rowbuf)[B], float (*colbuf)[B], int mode)
{
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll 1
    for (int k0 = 0; k0 < B; k0 += 4) {
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            const int k = k0 + kk, buf = k & 1;
            if (mode != 2 && ty == (k >> 2))   // row k of s: its owners are the threads of row block k/4
                *(float4*)&rowbuf[buf][tx * 4] = make_float4(acc[kk][0], acc[kk][1], acc[kk][2], acc[kk][3]);
            if (mode != 1 && tx == (k >> 2))   // column k of s
                *(float4*)&colbuf[buf][ty * 4] = make_float4(acc[0][kk], acc[1][kk], acc[2][kk], acc[3][kk]);
            __syncthreads();
            const float4 a = mode == 1 ? *(const float4*)&dgT[k][ty * 4] : *(const float4*)&colbuf[buf][ty * 4];
            const float4 b = mode == 2 ? *(const float4*)&dg[k][tx * 4] : *(const float4*)&rowbuf[buf][tx * 4];
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fminf(acc[r][c], av[r] + bv[c]);
        }
    }
}

// min(a, b, c) in one instruction (sm_100)
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ void tile_load(float (&acc)[4][4], const float* src, int ld)
{
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const float4 v = *(const float4*)(src + (long long)(ty * 4 + r) * ld + tx * 4);
        acc[r][0] = v.x; acc[r][1] = v.y; acc[r][2] = v.z; acc[r][3] = v.w;
    }
}

__device__ __forceinline__ void tile_store(float* dst, int ld, const float (&acc)[4][4])
{
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
    for (int r = 0; r < 4; r++)
        *(float4*)(dst + (long long)(ty * 4 + r) * ld + tx * 4) = make_float4(acc[r][0], acc[r][1], acc[r][2], acc[r][3]);
}

// A 64 x 64 block into shared memory, row-major (rm) and/or transposed (tr).
// Thread q reads the 4 floats at row q % 64, columns 4 (q / 64) + 16 it..:
// a warp covers 32 consecutive rows of one column group, so the transposed
// stores of a warp hit 32 consecutive words (no bank conflict).
__device__ __forceinline__ void block_to_smem(const float* src, int ld, float (*rm)[B + 4], float (*tr)[B + 4])
{
#pragma unroll
    for (int it = 0; it < B * B / 4 / FW_THREADS; it++) {
        const int q = threadIdx.x + it * FW_THREADS;
        const int i = q & (B - 1), j4 = (q >> 6) << 2;
        const float4 v = *(const float4*)(src + (long long)i * ld + j4);
        if (rm) *(float4*)&rm[i][j4] = v;
        if (tr) {
            tr[j4][i] = v.x; tr[j4 + 1][i] = v.y; tr[j4 + 2][i] = v.z; tr[j4 + 3][i] = v.w;
        }
    }
}

struct __align__(16) FwSmem {
    union {
        struct {
            float dg[B][B + 4];     // the closed diagonal block, row-major
            float dgT[B][B + 4];    // and transposed
            float rowbuf[2][B];     // row k of the tile being closed
            float colbuf[2][B];     // column k
        } panel;
        struct {
            float at[B][B + 4];     // the (bi, kb) block transposed: at[k][i]
            float bk[B][B + 4];     // the (kb, bj) block: bk[k][j]
        } prod;
        double row[ONNELA_MAX_N];  // Onnela: the node's row, dense
    };
    double red[FW_THREADS / 32];
};

__device__ __forceinline__ void fw_batch_body(const FwBatch& p)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ FwSmem sm;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    // ---- A: +inf matrices with a zero diagonal; weight maxima
    for (int gi = 0; gi < p.ng; gi++) {
        const FWGraph g = p.gs[gi];
        const long long tot4 = (long long)g.np * g.np / 4;
        float4* d = (float4*)(p.D + g.off);
        for (long long q = tid; q < tot4; q += nt) {
            const long long e = q * 4, i = e / g.np, j = e % g.np;
            float4 v = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
            if (i >= j && i < j + 4) ((float*)&v)[i - j] = 0.0f;
            d[q] = v;
        }
    }
    if (p.onnela) {
        for (int gi = blockIdx.x; gi < p.ng; gi += gridDim.x) {
            const FWGraph g = p.gs[gi];
            const int32_t nnz = g.R[g.n];
            float m = -INFINITY;
            for (int32_t q = threadIdx.x; q < nnz; q += FW_THREADS) m = fmaxf(m, g.V[q]);
            for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            __shared__ float mx[FW_THREADS / 32];
            if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = m;
            __syncthreads();
            if (threadIdx.x == 0) {
                float t = -INFINITY;
                for (int w = 0; w < FW_THREADS / 32; w++) t = fmaxf(t, mx[w]);
                p.vmax[gi] = t;
            }
            __syncthreads();
        }
    }
    grid.sync();
    // ---- B: edge distances 1/w (init_block, FormBlock.cpp:64); per-edge cube
    // roots of the normalised weights for Onnela
    for (int gi = 0; gi < p.ng; gi++) {
        const FWGraph g = p.gs[gi];
        const long long warps = nt >> 5;
        const float vm = p.onnela ? p.vmax[gi] : 1.0f;
        const long long e0 = p.onnela ? p.edge0[gi] : 0;
        for (long long i = tid >> 5; i < g.n; i += warps)
            for (int32_t q = g.R[i] + (threadIdx.x & 31); q < g.R[i + 1]; q += 32) {
                const int j = g.C[q];
                if (p.onnela) p.cw[e0 + q] = cbrt((double)__fdiv_rn(g.V[q], vm));
                if (j == i) continue;
                p.D[g.off + i * g.np + j] = g.V ? __fdiv_rn(1.0f, g.V[q]) : 1.0f;
            }
    }
    if (p.onnela) {
        grid.sync();
        for (int q = threadIdx.x; q < ONNELA_MAX_N; q += FW_THREADS) sm.row[q] = 0.0;
        __shared__ int s_x;
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0) s_x = atomicAdd(p.onnela_next, 1);
            __syncthreads();
            const int x = s_x;
            if (x >= p.total_nodes) break;
            onnela_node(p, x, sm.row, sm.red);
        }
    }
    grid.sync();
    // ---- FW rounds over all graphs with more than kb blocks
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    for (int kb = 0; kb < p.max_nb; kb++) {
        const int act = p.active[kb];
        // 1: diagonal blocks
        for (int gi = blockIdx.x; gi < act; gi += gridDim.x) {
            const FWGraph g = p.gs[gi];
            float* d = blk(p.D, g, kb, kb);
            float acc[4][4];
            tile_load(acc, d, g.np);
            closure(acc, sm.panel.dg, sm.panel.dgT, sm.panel.rowbuf, sm.panel.colbuf, 0);
            tile_store(d, g.np, acc);
            __syncthreads();
        }
        grid.sync();
        // 2: row and column panels
        const long long n2 = p.p2[act];
        for (long long t = blockIdx.x; t < n2; t += gridDim.x) {
            const int gi = task_graph(p.p2, act, t);
            const FWGraph g = p.gs[gi];
            const int local = (int)(t - p.p2[gi]);
            const bool row = local < g.nb - 1;
            int other = row ? local : local - (g.nb - 1);
            if (other >= kb) other++;
            float* d = row ? blk(p.D, g, kb, other) : blk(p.D, g, other, kb);
            block_to_smem(blk(p.D, g, kb, kb), g.np, row ? nullptr : sm.panel.dg, row ? sm.panel.dgT : nullptr);
            float acc[4][4];
            tile_load(acc, d, g.np);
            __syncthreads();
            closure(acc, sm.panel.dg, sm.panel.dgT, sm.panel.rowbuf, sm.panel.colbuf, row ? 1 : 2);
            tile_store(d, g.np, acc);
            __syncthreads();
        }
        grid.sync();
        // 3: the other blocks, register-tiled min-plus
        const long long n3 = p.p3[act];
        for (long long t = blockIdx.x; t < n3; t += gridDim.x) {
            const int gi = task_graph(p.p3, act, t);
            const FWGraph g = p.gs[gi];
            const int m = g.nb - 1;
            const int local = (int)(t - p.p3[gi]);
            int bi = local / m, bj = local % m;
            if (bi >= kb) bi++;
            if (bj >= kb) bj++;
            block_to_smem(blk(p.D, g, bi, kb), g.np, nullptr, sm.prod.at);
            block_to_smem(blk(p.D, g, kb, bj), g.np, sm.prod.bk, nullptr);
            float* c = blk(p.D, g, bi, bj);
            float acc[4][4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const float4 v = *(const float4*)(c + (long long)(ty * 4 + r) * g.np + tx * 4);
                acc[r][0] = v.x; acc[r][1] = v.y; acc[r][2] = v.z; acc[r][3] = v.w;
            }
            __syncthreads();
            // two k per step through the three-input minimum: one ALU
            // instruction per two updates (the min-plus is bound by that
            // pipe); min is exact, so the result equals the one-k loop's
#pragma unroll 4
            for (int k = 0; k < B; k += 2) {
                const float4 ai = *(const float4*)&sm.prod.at[k][ty * 4];
                const float4 bj4 = *(const float4*)&sm.prod.bk[k][tx * 4];
                const float4 ai1 = *(const float4*)&sm.prod.at[k + 1][ty * 4];
                const float4 bj1 = *(const float4*)&sm.prod.bk[k + 1][tx * 4];
                const float av[4] = {ai.x, ai.y, ai.z, ai.w}, av1[4] = {ai1.x, ai1.y, ai1.z, ai1.w};
                const float bv[4] = {bj4.x, bj4.y, bj4.z, bj4.w}, bv1[4] = {bj1.x, bj1.y, bj1.z, bj1.w};
#pragma unroll
                for (int r = 0; r < 4; r++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[r][q] = min3f(acc[r][q], av[r] + bv[q], av1[r] + bv1[q]);
            }
#pragma unroll
            for (int r = 0; r < 4; r++)
                *(float4*)(c + (long long)(ty * 4 + r) * g.np + tx * 4) =
                    make_float4(acc[r][0], acc[r][1], acc[r][2], acc[r][3]);
            __syncthreads();
        }
        grid.sync();
    }
    // ---- C: row sums of 1/d over finite, non-tiny distances (CUBFW_Lp.cpp:77-83,99-104)
    {
        const int lane = threadIdx.x & 31;
        const long long warps = nt >> 5;
        for (long long x = tid >> 5; x < p.total_nodes; x += warps) {
            const int gi = p.node_graph[x];
            const FWGraph g = p.gs[gi];
            const int u = (int)x - g.node0;
            const float* row = p.D + g.off + (long long)u * g.np;
            double acc = 0.0;
            for (int v = lane; v < g.n; v += 32) {
                const float d = row[v];
                if (v == u || !(d >= 0.1f)) continue;
                acc += 1.0 / (double)d;
            }
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) {
                p.rowsum[x] = acc;
                float e = g.n > 1 ? (float)(acc / (double)(g.n - 1)) : 0.0f;
                if (e < 1.0f / (float)g.n) e = 0.0f;
                p.eff[x] = e;
            }
        }
    }
    grid.sync();
    for (long long gi = tid; gi < p.ng; gi += nt) {
        const FWGraph g = p.gs[gi];
        double t = 0.0;
        for (int u = 0; u < g.n; u++) t += p.rowsum[g.node0 + u];
        p.lp[gi] = t > 0.0 ? 1.0 / (t / g.n / (g.n - 1)) : INFINITY;
        if (p.onnela) {
            double c = 0.0;
            for (int u = 0; u < g.n; u++) c += (double)p.cp[g.node0 + u];
            p.cp_mean[gi] = g.n > 0 ? c / g.n : 0.0;
        }
    }
}

// The kernel under two register budgets (2 or 4 resident CTAs per SM); the
// autotuner times both on the real batch (same arithmetic, same results).
template <int MINB>
__global__ void __launch_bounds__(FW_THREADS, MINB) k_fw_batch(FwBatch p)
{
    fw_batch_body(p);
}

__global__ void k_fw_copy_out(const FWGraph* __restrict__ gs, const float* __restrict__ D, float* __restrict__ out)
{
    const FWGraph g = gs[0];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)g.n * g.n;
         q += (long long)gridDim.x * blockDim.x)
        out[q] = D[g.off + (q / g.n) * g.np + q % g.n];
}

// outputs in processing order -> caller's order
__global__ void k_fw_unpermute(const int* __restrict__ perm, const FWGraph* __restrict__ gs, int ng,
                               const int* __restrict__ node0_out, const float* __restrict__ eff,
                               const double* __restrict__ lp, const float* __restrict__ cp,
                               const double* __restrict__ cpm, float* __restrict__ eff_o, double* __restrict__ lp_o,
                               float* __restrict__ cp_o, double* __restrict__ cpm_o, int onnela)
{
    for (int gi = blockIdx.x; gi < ng; gi += gridDim.x) {
        const FWGraph g = gs[gi];
        const int dst = perm[gi];
        const int o = node0_out[dst];
        for (int u = threadIdx.x; u < g.n; u += blockDim.x) {
            eff_o[o + u] = eff[g.node0 + u];
            if (onnela) cp_o[o + u] = cp[g.node0 + u];
        }
        if (threadIdx.x == 0) {
            lp_o[dst] = lp[gi];
            if (onnela) cpm_o[dst] = cpm[gi];
        }
    }
}
}  // namespace

// Graph table in processing order and the device batch description.
struct FwPlan {
    FwBatch b;
    FWGraph* dtab;
    int* perm;          // processing index -> caller's index
    int* node0_out;     // caller's node offsets
    long long total;
    int grid;
    int minb;           // register budget of the kernel instance (resident CTAs per SM)
};

static pg_status fw_launch(pg_ctx* ctx, FwPlan* P, bool profiled);

static pg_status fw_plan(pg_ctx* ctx, const pg_graph* const* graphs, int ng, bool onnela, FwPlan* P)
{
    std::vector<int> order(ng);
    std::iota(order.begin(), order.end(), 0);
    auto nb_of = [&](int i) { return std::max(1, (graphs[i]->n + B - 1) / B); };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return nb_of(x) > nb_of(y); });
    std::vector<FWGraph> tab(ng);
    std::vector<long long> p2(ng + 1, 0), p3(ng + 1, 0), edge0(ng, 0);
    long long edges = 0;
    std::vector<int> perm(ng), node0_out(ng), node_graph;
    long long off = 0;
    int node0 = 0, nmax = 1, max_nb = 0;
    int o = 0;
    for (int i = 0; i < ng; i++) {
        node0_out[i] = o;
        o += graphs[i]->n;
    }
    for (int q = 0; q < ng; q++) {
        const pg_graph* g = graphs[order[q]];
        if (onnela && !g->V) return pg_fail(ctx, PG_ERR_INVALID, "Onnela clustering needs a weighted graph");
        const int nb = nb_of(order[q]);
        tab[q] = {g->R, g->C, g->V, g->n, nb * B, nb, off, node0};
        perm[q] = order[q];
        off += (long long)nb * B * nb * B;
        for (int u = 0; u < g->n; u++) node_graph.push_back(q);
        node0 += g->n;
        nmax = std::max(nmax, (int)g->n);
        max_nb = std::max(max_nb, nb);
        edge0[q] = edges;
        edges += g->nnz;
        p2[q + 1] = p2[q] + 2LL * (nb - 1);
        p3[q + 1] = p3[q] + (long long)(nb - 1) * (nb - 1);
    }
    if (onnela && nmax > ONNELA_MAX_N)
        return pg_fail(ctx, PG_ERR_TOO_LARGE, "Onnela in the batched launch: n=%d above %d", nmax, ONNELA_MAX_N);
    std::vector<int> active(max_nb);
    for (int kb = 0; kb < max_nb; kb++) {
        int a = 0;
        while (a < ng && tab[a].nb > kb) a++;
        active[kb] = a;
    }
    FwBatch& b = P->b;
    memset(&b, 0, sizeof b);
    int *dact, *dng, *dperm, *dn0;
    long long *dp2, *dp3, *de0;
    PG_TRY(pg_wst(ctx, "fw.D", (size_t)off, &b.D));
    PG_TRY(pg_wst(ctx, "fw.tab", (size_t)ng, &P->dtab));
    PG_TRY(pg_wst(ctx, "fw.active", (size_t)max_nb, &dact));
    PG_TRY(pg_wst(ctx, "fw.p2", (size_t)ng + 1, &dp2));
    PG_TRY(pg_wst(ctx, "fw.p3", (size_t)ng + 1, &dp3));
    PG_TRY(pg_wst(ctx, "fw.edge0", (size_t)ng, &de0));
    PG_TRY(pg_wst(ctx, "fw.cw", (size_t)(onnela ? edges : 0) + 1, &b.cw));
    PG_TRY(pg_wst(ctx, "fw.ngraph", (size_t)node0 + 1, &dng));
    PG_TRY(pg_wst(ctx, "fw.perm", (size_t)ng, &dperm));
    PG_TRY(pg_wst(ctx, "fw.node0o", (size_t)ng, &dn0));
    PG_TRY(pg_wst(ctx, "fw.vmax", (size_t)ng, &b.vmax));
    PG_TRY(pg_wst(ctx, "fw.next", 1, &b.onnela_next));
    PG_TRY(pg_wst(ctx, "fw.rows", (size_t)node0 + 1, &b.rowsum));
    PG_TRY(pg_wst(ctx, "fw.eff", (size_t)node0 + 1, &b.eff));
    PG_TRY(pg_wst(ctx, "fw.lp", (size_t)ng, &b.lp));
    PG_TRY(pg_wst(ctx, "fw.cp", (size_t)node0 + 1, &b.cp));
    PG_TRY(pg_wst(ctx, "fw.cpm", (size_t)ng, &b.cp_mean));
    PG_CUDA(ctx, cudaMemcpyAsync(P->dtab, tab.data(), sizeof(FWGraph) * ng, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(dact, active.data(), sizeof(int) * max_nb, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(dp2, p2.data(), sizeof(long long) * (ng + 1), cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(dp3, p3.data(), sizeof(long long) * (ng + 1), cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(de0, edge0.data(), sizeof(long long) * ng, cudaMemcpyHostToDevice, ctx->stream));
    if (node0 > 0)
        PG_CUDA(ctx, cudaMemcpyAsync(dng, node_graph.data(), sizeof(int) * node0, cudaMemcpyHostToDevice,
                                     ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(dperm, perm.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(dn0, node0_out.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // host tables' lifetime
    b.gs = P->dtab;
    b.ng = ng;
    b.total_nodes = node0;
    b.max_nb = max_nb;
    b.active = dact;
    b.p2 = dp2;
    b.p3 = dp3;
    b.edge0 = de0;
    b.node_graph = dng;
    b.onnela = onnela;
    P->perm = dperm;
    P->node0_out = dn0;
    P->total = node0;
    int per2 = 0, per4 = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_fw_batch<2>, FW_THREADS, 0));
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per4, k_fw_batch<4>, FW_THREADS, 0));
    if (per2 < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "FW: kernel does not fit an SM");
    // choices: (register budget, resident CTAs per SM)
    std::vector<TuneChoice> cands;
    for (int c = 1; c <= std::min(per2, 2); c++) cands.push_back({2, c});
    for (int c = 3; c <= std::min(per4, 4); c++) cands.push_back({4, c});
    TuneChoice best{2, std::min(per2, 2)};
    // shape bucket: log2 of the rms padded graph size and log2 of the number
    // of graphs (passed as the "mean degree" of the key); a 160- and a
    // 512-graph batch of the same sizes must not share a choice
    const long long rms = off > 0 ? (long long)std::sqrt((double)off / ng) : 0;
    const std::string key = tune_key("fw_batch", rms, (long long)ng * std::max(1LL, rms));
    PG_TRY(tune_pick(ctx, key, cands, &best, [&](const TuneChoice& c) -> pg_status {
        P->minb = c.a;
        P->grid = ctx->sm_count * c.b;
        return fw_launch(ctx, P, false);
    }));
    P->minb = best.a;
    P->grid = ctx->sm_count * best.b;
    return PG_OK;
}

static pg_status fw_launch(pg_ctx* ctx, FwPlan* P, bool profiled)
{
    PG_CUDA(ctx, cudaMemsetAsync(P->b.onnela_next, 0, sizeof(int), ctx->stream));
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeCooperative;
    attr.val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P->grid);
    cfg.blockDim = dim3(FW_THREADS);
    cfg.stream = ctx->stream;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    const int h = profiled ? pg_prof_begin(ctx, "k_fw_batch") : -1;
    if (P->minb == 4) PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_fw_batch<4>, P->b));
    else PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_fw_batch<2>, P->b));
    PG_LAUNCHED(ctx);
    pg_prof_end(ctx, h);
    return PG_OK;
}

extern "C" pg_status pg_fw_paths(pg_ctx* ctx, const pg_graph* g, float* dist, float* eff, double* lp)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_fw_paths: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    const pg_graph* one[1] = {g};
    FwPlan P;
    PG_TRY(fw_plan(ctx, one, 1, false, &P));
    PG_TRY(fw_launch(ctx, &P, true));
    if (dist) {
        float* tmp;
        PG_TRY(pg_wst(ctx, "fw.out", (size_t)n * n + 1, &tmp));
        k_fw_copy_out<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(P.dtab, P.b.D, tmp);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_d2h(ctx, dist, tmp, sizeof(float) * (size_t)n * n));
    }
    if (eff) PG_TRY(pg_d2h(ctx, eff, P.b.eff, sizeof(float) * n));
    if (lp) PG_TRY(pg_d2h(ctx, lp, P.b.lp, sizeof(double)));
    return PG_OK;
}

extern "C" pg_status pg_fw_batched(pg_ctx* ctx, const pg_graph* const* graphs, int32_t count, float* eff, double* lp,
                                   float* cp, double* cp_mean)
{
    if (!ctx || !graphs || count < 1) return pg_fail(ctx, PG_ERR_INVALID, "pg_fw_batched: bad arguments");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    for (int i = 0; i < count; i++)
        if (!graphs[i]) return pg_fail(ctx, PG_ERR_INVALID, "graph %d is null", i);
    const bool onnela = cp || cp_mean;
    FwPlan P;
    PG_TRY(fw_plan(ctx, graphs, count, onnela, &P));
    PG_TRY(fw_launch(ctx, &P, true));
    float *deff, *dcp;
    double *dlp, *dcpm;
    PG_TRY(pg_wst(ctx, "fwb.eff", (size_t)P.total + 1, &deff));
    PG_TRY(pg_wst(ctx, "fwb.cp", (size_t)P.total + 1, &dcp));
    PG_TRY(pg_wst(ctx, "fwb.lp", (size_t)count, &dlp));
    PG_TRY(pg_wst(ctx, "fwb.cpm", (size_t)count, &dcpm));
    k_fw_unpermute<<<std::min(count, 4096), 256, 0, ctx->stream>>>(P.perm, P.dtab, count, P.node0_out, P.b.eff, P.b.lp,
                                                                   P.b.cp, P.b.cp_mean, deff, dlp, dcp, dcpm,
                                                                   onnela);
    PG_LAUNCHED(ctx);
    if (eff) PG_TRY(pg_d2h(ctx, eff, deff, sizeof(float) * P.total));
    if (lp) PG_TRY(pg_d2h(ctx, lp, dlp, sizeof(double) * count));
    if (cp) PG_TRY(pg_d2h(ctx, cp, dcp, sizeof(float) * P.total));
    if (cp_mean) PG_TRY(pg_d2h(ctx, cp_mean, dcpm, sizeof(double) * count));
    return PG_OK;
}
