// pc.cu -- participation coefficient of every node from module labels, as the
// reference's PC_CPU (W/PC_CPU/PC_CPU/main.cpp:100-174), in float arithmetic
// with the reference's order of operations, so results are bit-identical:
//   strength s_i = the row's weights added in row order;
//   w_im = the row's weights towards module m, added in row order;
//   PC_i = 1 - sum over m = 1..K in order of (w_im / s_i)^2, 0 when s_i = 0;
//   normalised PC_i = PC_i / ((K - 1) / K) unless K = 1.
// One warp per node.  Lane l keeps the sums of the modules m with
// (m - 1) % 32 == l in the warp's slice of shared memory, so every module's
// sum is built in row order by a single lane; lane 0 then forms the sum over
// modules in order.  Explicit _rn intrinsics keep the compiler from fusing
// multiplies and adds, which the reference's build does not do.
#include "pg_internal.cuh"
#include <algorithm>

namespace {
constexpr int PC_THREADS = 256;

__global__ void __launch_bounds__(PC_THREADS)
k_pc(const int32_t* __restrict__ R, const int32_t* __restrict__ C, const float* __restrict__ V, int n,
     const float* __restrict__ module, int K, float mx, float* __restrict__ acc_global, float* __restrict__ pc,
     float* __restrict__ pc_norm)
{
    extern __shared__ float acc_shared[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    float* acc = acc_global ? acc_global + (size_t)gw * K : acc_shared + (size_t)wib * K;
    for (int v = gw; v < n; v += nw) {
        const int e0 = R[v], e1 = R[v + 1];
        float deg = 0.0f;
        for (int j = e0; j < e1; j++) deg = __fadd_rn(deg, V ? V[j] : 1.0f);
        float p = 0.0f;
        if (deg != 0.0f) {
            for (int m = lane; m < K; m += 32) acc[m] = 0.0f;
            __syncwarp();
            for (int j = e0; j < e1; j++) {
                const int m = (int)module[C[j]] - 1;
                if (m >= 0 && (m & 31) == lane) acc[m] = __fadd_rn(acc[m], V ? V[j] : 1.0f);
            }
            __syncwarp();
            if (lane == 0) {
                float sum = 0.0f;
                for (int m = 0; m < K; m++) {
                    const float t = __fdiv_rn(acc[m], deg);
                    sum = __fadd_rn(sum, __fmul_rn(t, t));
                }
                p = __fsub_rn(1.0f, sum);
            }
            __syncwarp();   // the sums are read before the next node clears them
        }
        if (lane == 0) {
            pc[v] = p;
            pc_norm[v] = K != 1 ? __fdiv_rn(p, mx) : p;
        }
    }
}
}  // namespace

extern "C" pg_status pg_participation(pg_ctx* ctx, const pg_graph* g, const float* module, float* pc, float* pc_norm,
                                      int32_t* n_modules)
{
    if (!ctx || !g || !module || !pc || !pc_norm) return pg_fail(ctx, PG_ERR_INVALID, "pg_participation: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    int K = 0;
    for (int i = 0; i < n; i++) K = std::max(K, (int)module[i]);
    if (n_modules) *n_modules = K;
    if (n == 0) return PG_OK;
    const float mx = K != 1 ? (float)(K - 1) / (float)K : 1.0f;
    float *dmod, *dpc, *dpn, *gacc = nullptr;
    PG_TRY(pg_wst(ctx, "pc.module", (size_t)n, &dmod));
    PG_TRY(pg_wst(ctx, "pc.pc", (size_t)n, &dpc));
    PG_TRY(pg_wst(ctx, "pc.norm", (size_t)n, &dpn));
    PG_CUDA(ctx, cudaMemcpyAsync(dmod, module, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    const int Kc = std::max(K, 1);
    const int grid = ctx->sm_count * 8;
    // module sums in shared memory when the block's eight warps fit, else in
    // a global slice per warp
    size_t smem = (size_t)(PC_THREADS / 32) * Kc * sizeof(float);
    const size_t cap = (size_t)ctx->smem_optin - 4096;
    if (smem > cap) {
        PG_TRY(pg_wst(ctx, "pc.acc", (size_t)grid * (PC_THREADS / 32) * Kc, &gacc));
        smem = 0;
    } else if (smem > 48 * 1024) {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_pc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    k_pc<<<grid, PC_THREADS, smem, ctx->stream>>>(g->R, g->C, g->V, n, dmod, Kc, mx, gacc, dpc, dpn);
    PG_LAUNCHED(ctx);
    PG_TRY(pg_d2h(ctx, pc, dpc, sizeof(float) * n));
    PG_TRY(pg_d2h(ctx, pc_norm, dpn, sizeof(float) * n));
    return PG_OK;
}
