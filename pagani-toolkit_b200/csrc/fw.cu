// fw.cu -- weighted path length by blocked Floyd-Warshall in FP32 min-plus
// (CUBFW_Lp, W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp.cpp:13-162; phases of cuAPSP,
// CUBFW.cpp:19-168 and BFW_C, BFW.cpp:40-109) for one graph or a batch of
// graphs in grouped launches.
//
// Every graph's dense distance matrix stays in HBM for the whole sweep
// (the reference streamed 3072^2 blocks over PCIe per phase).  Matrices are
// padded to a multiple of the 32x32 block; block k of every graph is
// processed by the same three launches (diagonal block, its row and column
// panels, the rest), so a batch of 512 graphs needs 3 launches per k step.
#include "pg_internal.cuh"
#include <cmath>
#include <algorithm>

pg_status pg_onnela_table(pg_ctx* ctx, const pg_graph* const* graphs, int ng, int first_n, float* cp_dev,
                          double* mean_dev);

namespace {
constexpr int B = 32;

struct FWGraph {
    const int32_t* R;
    const int32_t* C;
    const float* V;     // null: every edge has distance 1
    int32_t n, np, nb;  // nodes, padded size, blocks per side
    long long off;      // matrix offset (elements)
    int32_t node0;      // offset of its nodes in concatenated outputs
};

__global__ void k_fw_fill(const FWGraph* __restrict__ gs, int ng, float* __restrict__ D)
{
    const FWGraph g = gs[blockIdx.y];
    const long long tot = (long long)g.np * g.np;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
        long long i = q / g.np, j = q % g.np;
        D[g.off + q] = (i == j) ? 0.0f : INFINITY;
    }
}

// Edge distances 1/w (init_block, FormBlock.cpp:64); diagonal stays 0.
__global__ void k_fw_edges(const FWGraph* __restrict__ gs, int ng, float* __restrict__ D)
{
    const FWGraph g = gs[blockIdx.y];
    for (int i = blockIdx.x; i < g.n; i += gridDim.x)
        for (int32_t q = g.R[i] + threadIdx.x; q < g.R[i + 1]; q += blockDim.x) {
            int j = g.C[q];
            if (j == i) continue;
            float d = g.V ? __fdiv_rn(1.0f, g.V[q]) : 1.0f;
            D[g.off + (long long)i * g.np + j] = d;
        }
}

__device__ __forceinline__ float* blk(float* D, const FWGraph& g, int bi, int bj)
{
    return D + g.off + (long long)bi * B * g.np + (long long)bj * B;
}

// Phase 1: closure of the diagonal block kb.
__global__ void k_fw_ph1(const FWGraph* __restrict__ gs, float* __restrict__ D, int kb)
{
    const FWGraph g = gs[blockIdx.y];
    if (kb >= g.nb) return;
    __shared__ float s[B][B + 1];
    const int ty = threadIdx.y, tx = threadIdx.x;
    float* p = blk(D, g, kb, kb);
    s[ty][tx] = p[(long long)ty * g.np + tx];
    __syncthreads();
    for (int k = 0; k < B; k++) {
        float c = s[ty][k] + s[k][tx];
        __syncthreads();
        if (c < s[ty][tx]) s[ty][tx] = c;
        __syncthreads();
    }
    p[(long long)ty * g.np + tx] = s[ty][tx];
}

// Phase 2: row panel (kb, j) and column panel (i, kb) against the closed
// diagonal block, in place inside the panel block as BFW_one_block_C does.
__global__ void k_fw_ph2(const FWGraph* __restrict__ gs, float* __restrict__ D, int kb)
{
    const FWGraph g = gs[blockIdx.y];
    if (kb >= g.nb) return;
    int idx = blockIdx.x;
    if (idx >= 2 * (g.nb - 1)) return;
    const bool row = idx < g.nb - 1;
    int other = row ? idx : idx - (g.nb - 1);
    if (other >= kb) other++;
    __shared__ float dg[B][B + 1];
    __shared__ float s[B][B + 1];
    const int ty = threadIdx.y, tx = threadIdx.x;
    float* pd = blk(D, g, kb, kb);
    float* p = row ? blk(D, g, kb, other) : blk(D, g, other, kb);
    dg[ty][tx] = pd[(long long)ty * g.np + tx];
    s[ty][tx] = p[(long long)ty * g.np + tx];
    __syncthreads();
    for (int k = 0; k < B; k++) {
        float c = row ? dg[ty][k] + s[k][tx] : s[ty][k] + dg[k][tx];
        __syncthreads();
        if (c < s[ty][tx]) s[ty][tx] = c;
        __syncthreads();
    }
    p[(long long)ty * g.np + tx] = s[ty][tx];
}

// Phase 3: every other block (i, j) = min(d_ij, d_i,kb (x) d_kb,j).
__global__ void k_fw_ph3(const FWGraph* __restrict__ gs, float* __restrict__ D, int kb)
{
    const FWGraph g = gs[blockIdx.y];
    if (kb >= g.nb) return;
    const int m = g.nb - 1;
    int idx = blockIdx.x;
    if (idx >= m * m) return;
    int bi = idx / m, bj = idx % m;
    if (bi >= kb) bi++;
    if (bj >= kb) bj++;
    __shared__ float a[B][B + 1];
    __shared__ float b[B][B + 1];
    const int ty = threadIdx.y, tx = threadIdx.x;
    a[ty][tx] = blk(D, g, bi, kb)[(long long)ty * g.np + tx];
    b[ty][tx] = blk(D, g, kb, bj)[(long long)ty * g.np + tx];
    __syncthreads();
    float* p = blk(D, g, bi, bj) + (long long)ty * g.np + tx;
    float cur = *p;
#pragma unroll
    for (int k = 0; k < B; k++) cur = fminf(cur, a[ty][k] + b[k][tx]);
    *p = cur;
}

// Row sums of 1/d over finite, non-tiny distances (CUBFW_Lp.cpp:77-83,99-104).
__global__ void k_fw_rows(const FWGraph* __restrict__ gs, int ng, const float* __restrict__ D,
                          double* __restrict__ rowsum, float* __restrict__ eff)
{
    const FWGraph g = gs[blockIdx.y];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int u = blockIdx.x * nw + w; u < g.n; u += gridDim.x * nw) {
        const float* row = D + g.off + (long long)u * g.np;
        double acc = 0.0;
        for (int v = lane; v < g.n; v += 32) {
            float x = row[v];
            if (v == u || !(x >= 0.1f)) continue;
            acc += 1.0 / (double)x;
        }
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            rowsum[g.node0 + u] = acc;
            float e = g.n > 1 ? (float)(acc / (double)(g.n - 1)) : 0.0f;
            if (e < 1.0f / (float)g.n) e = 0.0f;
            eff[g.node0 + u] = e;
        }
    }
}

__global__ void k_fw_lp(const FWGraph* __restrict__ gs, int ng, const double* __restrict__ rowsum,
                        double* __restrict__ lp)
{
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += gridDim.x * blockDim.x) {
        const FWGraph g = gs[gi];
        double t = 0.0;
        for (int u = 0; u < g.n; u++) t += rowsum[g.node0 + u];
        lp[gi] = t > 0.0 ? 1.0 / (t / g.n / (g.n - 1)) : INFINITY;
    }
}

__global__ void k_fw_copy_out(const FWGraph* __restrict__ gs, const float* __restrict__ D, float* __restrict__ out)
{
    const FWGraph g = gs[0];
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < (long long)g.n * g.n;
         q += (long long)gridDim.x * blockDim.x)
        out[q] = D[g.off + (q / g.n) * g.np + q % g.n];
}
}  // namespace

static pg_status fw_run(pg_ctx* ctx, const pg_graph* const* graphs, int ng, float* eff_dev, double* lp_dev,
                        float** dist_dev_out, FWGraph** tab_out)
{
    std::vector<FWGraph> tab(ng);
    long long off = 0;
    int node0 = 0, nbmax = 0;
    for (int i = 0; i < ng; i++) {
        const pg_graph* g = graphs[i];
        int np = std::max(B, (g->n + B - 1) / B * B);
        tab[i] = {g->R, g->C, g->V, g->n, np, np / B, off, node0};
        off += (long long)np * np;
        node0 += g->n;
        nbmax = std::max(nbmax, np / B);
    }
    float* D;
    FWGraph* dtab;
    double* rowsum;
    PG_TRY(pg_wst(ctx, "fw.D", (size_t)off, &D));
    PG_TRY(pg_wst(ctx, "fw.tab", (size_t)ng, &dtab));
    PG_TRY(pg_wst(ctx, "fw.rows", (size_t)node0 + 1, &rowsum));
    PG_CUDA(ctx, cudaMemcpyAsync(dtab, tab.data(), sizeof(FWGraph) * ng, cudaMemcpyHostToDevice, ctx->stream));
    // grid.y carries the graph index (at most 65535 graphs per launch)
    if (ng > 65535) return pg_fail(ctx, PG_ERR_INVALID, "at most 65535 graphs per batch");
    k_fw_fill<<<dim3(64, ng), 256, 0, ctx->stream>>>(dtab, ng, D);
    PG_LAUNCHED(ctx);
    k_fw_edges<<<dim3(256, ng), 128, 0, ctx->stream>>>(dtab, ng, D);
    PG_LAUNCHED(ctx);
    for (int kb = 0; kb < nbmax; kb++) {
        k_fw_ph1<<<dim3(1, ng), dim3(B, B), 0, ctx->stream>>>(dtab, D, kb);
        PG_LAUNCHED(ctx);
        if (nbmax > 1) {
            k_fw_ph2<<<dim3(2 * (nbmax - 1), ng), dim3(B, B), 0, ctx->stream>>>(dtab, D, kb);
            PG_LAUNCHED(ctx);
            k_fw_ph3<<<dim3((nbmax - 1) * (nbmax - 1), ng), dim3(B, B), 0, ctx->stream>>>(dtab, D, kb);
            PG_LAUNCHED(ctx);
        }
    }
    k_fw_rows<<<dim3(std::max(1, std::min(1024, ceil_div(tab.empty() ? 1 : 1024, 8))), ng), 256, 0, ctx->stream>>>(
        dtab, ng, D, rowsum, eff_dev);
    PG_LAUNCHED(ctx);
    k_fw_lp<<<ceil_div(ng, 128), 128, 0, ctx->stream>>>(dtab, ng, rowsum, lp_dev);
    PG_LAUNCHED(ctx);
    if (dist_dev_out) *dist_dev_out = D;
    if (tab_out) *tab_out = dtab;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // host table lifetime
    return PG_OK;
}

extern "C" pg_status pg_fw_paths(pg_ctx* ctx, const pg_graph* g, float* dist, float* eff, double* lp)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_fw_paths: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    float* deff;
    double* dlp;
    PG_TRY(pg_wst(ctx, "fw.eff", (size_t)n + 1, &deff));
    PG_TRY(pg_wst(ctx, "fw.lp", 1, &dlp));
    const pg_graph* one[1] = {g};
    float* D;
    FWGraph* tab;
    PG_TRY(fw_run(ctx, one, 1, deff, dlp, &D, &tab));
    if (dist) {
        float* tmp;
        PG_TRY(pg_wst(ctx, "fw.out", (size_t)n * n + 1, &tmp));
        k_fw_copy_out<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(tab, D, tmp);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_d2h(ctx, dist, tmp, sizeof(float) * (size_t)n * n));
    }
    if (eff) PG_TRY(pg_d2h(ctx, eff, deff, sizeof(float) * n));
    if (lp) PG_TRY(pg_d2h(ctx, lp, dlp, sizeof(double)));
    return PG_OK;
}

extern "C" pg_status pg_fw_batched(pg_ctx* ctx, const pg_graph* const* graphs, int32_t count, float* eff, double* lp,
                                   float* cp, double* cp_mean)
{
    if (!ctx || !graphs || count < 1) return pg_fail(ctx, PG_ERR_INVALID, "pg_fw_batched: bad arguments");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    long long total = 0;
    for (int i = 0; i < count; i++) {
        if (!graphs[i]) return pg_fail(ctx, PG_ERR_INVALID, "graph %d is null", i);
        total += graphs[i]->n;
    }
    float *deff, *dcp;
    double *dlp, *dcpm;
    PG_TRY(pg_wst(ctx, "fwb.eff", (size_t)total + 1, &deff));
    PG_TRY(pg_wst(ctx, "fwb.lp", (size_t)count, &dlp));
    PG_TRY(fw_run(ctx, graphs, count, deff, dlp, nullptr, nullptr));
    if (cp || cp_mean) {
        PG_TRY(pg_wst(ctx, "fwb.cp", (size_t)total + 1, &dcp));
        PG_TRY(pg_wst(ctx, "fwb.cpm", (size_t)count, &dcpm));
        PG_TRY(pg_onnela_table(ctx, graphs, count, 0, dcp, dcpm));
        if (cp) PG_TRY(pg_d2h(ctx, cp, dcp, sizeof(float) * total));
        if (cp_mean) PG_TRY(pg_d2h(ctx, cp_mean, dcpm, sizeof(double) * count));
    }
    if (eff) PG_TRY(pg_d2h(ctx, eff, deff, sizeof(float) * total));
    if (lp) PG_TRY(pg_d2h(ctx, lp, dlp, sizeof(double) * count));
    return PG_OK;
}
