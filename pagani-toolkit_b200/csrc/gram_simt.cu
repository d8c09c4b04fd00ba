// gram_simt.cu -- plain FP32 Gram tiles on the SIMT pipes (the "FP32 GPU
// path"), fused with the threshold epilogue.  This is the FP32 counterpart of
// the reference's cublasSgemm tiles (U/CorMat/CUCorMat/CUCORMAT/CorMat.cu:93);
// nothing is written back except the kept pairs, the FP64 band and a
// histogram.
//
// Persistent CTAs walk the upper-triangle 128x128 tiles in row-major order
// (consecutive tiles share the row block in L2).  256 threads, 8x8 outputs
// per thread, K staged in 32-wide chunks through double-buffered shared
// memory with the next chunk prefetched into registers.
#include "build_graph.cuh"

namespace {
constexpr int BM = 128, BK = 32, PAD = 4, LDS = BM + PAD;
constexpr int THREADS = 256;
constexpr size_t SMEM_TILES = (size_t)2 * 2 * BK * LDS * sizeof(float);  // 2 stages x (A,B)

template <int MODE>
__global__ void __launch_bounds__(THREADS, 2)
k_gram_simt(const float* __restrict__ Z, int Tp, int nb, EpiParams p)
{
    extern __shared__ float smem[];
    float* As = smem;                       // [2][BK][LDS]
    float* Bs = smem + 2 * BK * LDS;        // [2][BK][LDS]
    unsigned int* sh_hist = (unsigned int*)(smem + 4 * BK * LDS);
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    if (MODE == EPI_HIST) {
        for (int b = t; b < HIST_BINS; b += THREADS) sh_hist[b] = 0;
        __syncthreads();
    }
    const long long nt = (long long)nb * (nb + 1) / 2;
    const int nk = Tp / BK;
    unsigned int below = 0u, neg = 0u;
    const long long stride = MODE == EPI_HIST ? (long long)p.tile_stride : 1LL;
    for (long long L = blockIdx.x * stride; L < nt; L += (long long)gridDim.x * stride) {
        int bi, bj;
        tri_tile(L, nb, bi, bj);
        const float* Ag = Z + (size_t)bi * BM * Tp;
        const float* Bg = Z + (size_t)bj * BM * Tp;
        float acc[8][8];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int b = 0; b < 8; b++) acc[a][b] = 0.0f;
        float4 ra[4], rb[4];
        auto gload = [&](int kc) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                int idx = t + THREADS * q, row = idx >> 3, c4 = idx & 7;
                ra[q] = *reinterpret_cast<const float4*>(Ag + (size_t)row * Tp + kc * BK + c4 * 4);
                rb[q] = *reinterpret_cast<const float4*>(Bg + (size_t)row * Tp + kc * BK + c4 * 4);
            }
        };
        auto sstore = [&](int st) {
            float* a = As + st * BK * LDS;
            float* b = Bs + st * BK * LDS;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                int idx = t + THREADS * q, row = idx >> 3, k = (idx & 7) * 4;
                a[(k + 0) * LDS + row] = ra[q].x; a[(k + 1) * LDS + row] = ra[q].y;
                a[(k + 2) * LDS + row] = ra[q].z; a[(k + 3) * LDS + row] = ra[q].w;
                b[(k + 0) * LDS + row] = rb[q].x; b[(k + 1) * LDS + row] = rb[q].y;
                b[(k + 2) * LDS + row] = rb[q].z; b[(k + 3) * LDS + row] = rb[q].w;
            }
        };
        gload(0);
        sstore(0);
        __syncthreads();
        for (int kc = 0; kc < nk; kc++) {
            const int st = kc & 1;
            if (kc + 1 < nk) gload(kc + 1);
            const float* a = As + st * BK * LDS + ty * 8;
            const float* b = Bs + st * BK * LDS + tx * 8;
#pragma unroll
            for (int k = 0; k < BK; k++) {
                float4 a0 = *reinterpret_cast<const float4*>(a + k * LDS);
                float4 a1 = *reinterpret_cast<const float4*>(a + k * LDS + 4);
                float4 b0 = *reinterpret_cast<const float4*>(b + k * LDS);
                float4 b1 = *reinterpret_cast<const float4*>(b + k * LDS + 4);
                float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                for (int x = 0; x < 8; x++)
#pragma unroll
                    for (int y = 0; y < 8; y++) acc[x][y] = fmaf(av[x], bv[y], acc[x][y]);
            }
            if (kc + 1 < nk) sstore(st ^ 1);
            __syncthreads();
        }
        // ---- fused threshold epilogue
        const int i0 = bi * BM + ty * 8, j0 = bj * BM + tx * 8;
        if (MODE == EPI_HIST) {
#pragma unroll
            for (int x = 0; x < 8; x++)
#pragma unroll
                for (int y = 0; y < 8; y++) {
                    int i = i0 + x, j = j0 + y;
                    if (i < j && j < p.N) epi_hist(acc[x][y], p, sh_hist, below, neg);
                }
        } else {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                unsigned int m1 = 0u, m2 = 0u;
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 8; y++) {
                        int i = i0 + 4 * h + x, j = j0 + y;
                        int cls = (i < j && j < p.N) ? epi_class(acc[4 * h + x][y], p) : 0;
                        m1 |= (unsigned)(cls == 1) << (x * 8 + y);
                        m2 |= (unsigned)(cls == 2) << (x * 8 + y);
                    }
                epi_emit_masks(m1, m2, p, [&](int q, int& i, int& j, float& r) {
                    int x = q >> 3, y = q & 7;
                    i = i0 + 4 * h + x;
                    j = j0 + y;
                    r = acc[4 * h + x][y];
                });
            }
        }
    }
    if (MODE == EPI_HIST) {
        epi_hist_flush(below, neg, p);
        __syncthreads();
        for (int b = t; b < HIST_BINS; b += THREADS)
            if (sh_hist[b]) atomicAdd(&p.hist[b], sh_hist[b]);
    }
}
}  // namespace

pg_status launch_gram_simt(pg_ctx* ctx, const ZOperands& z, int mode, const EpiParams& p)
{
    const int nb = z.Np / BM;
    const long long nt = (long long)nb * (nb + 1) / 2;
    size_t smem = SMEM_TILES + (mode == EPI_HIST ? HIST_BINS * sizeof(unsigned int) : 0);
    long long grid = 2LL * ctx->sm_count;
    if (grid > nt) grid = nt;
    if (mode == EPI_HIST) {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_gram_simt<EPI_HIST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_gram_simt<EPI_HIST><<<(int)grid, THREADS, smem, ctx->stream>>>(z.z32, z.Tp, nb, p);
    } else {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_gram_simt<EPI_EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        k_gram_simt<EPI_EMIT><<<(int)grid, THREADS, smem, ctx->stream>>>(z.z32, z.Tp, nb, p);
    }
    PG_LAUNCHED(ctx);
    return PG_OK;
}
