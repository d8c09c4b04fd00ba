// build_graph.cuh -- shared pieces of network construction: the operand
// layout in HBM and the fused threshold epilogue used by both Gram kernels
// (FP32 SIMT and tcgen05 split-BF16).
#pragma once
#include "pg_internal.cuh"

// Operands, all row-major with one row per voxel (the K = time dimension
// contiguous, i.e. "K-major" for both GEMM operands of Z * Z^T):
//   z64 : N  x T  double  -- exact z-scores for the FP64 recheck
//   z32 : Np x Tp float   -- rounded z-scores for the FP32 SIMT Gram
//   zhi : Np x Tp bf16    -- bf16(z32)
//   zlo : Np x Tp bf16    -- bf16(z32 - zhi)
// Np = N rounded up to the 128-row tile, Tp = T rounded up to 64; padding is 0.
struct ZOperands {
    int N, T, Np, Tp;
    double* z64;
    float* z32;
    __nv_bfloat16* zhi;
    __nv_bfloat16* zlo;
};

enum : int { EPI_HIST = 0, EPI_EMIT = 1 };
constexpr int HIST_BINS = 4096;

// Threshold epilogue parameters (keys are r, or |r| in ABS mode).
struct EpiParams {
    int N;
    int abs_mode;
    int weighted;
    // HIST: bin = clamp((key - kmin) * scale)
    float kmin, scale;
    unsigned int* hist;            // HIST_BINS global counters
    // EMIT: key >= hi_cut -> decided edge; key >= lo_cut -> FP64 band;
    // |r| >= edge_band -> band (range rule near +-1).
    float lo_cut, hi_cut, edge_band;
    int2* pairs;                   // decided edges (i < j)
    float* pair_w;                 // their weights (weighted only)
    unsigned long long* n_pairs;
    long long cap_pairs;
    int2* band;                    // band pairs (i < j)
    unsigned long long* n_band;
    long long cap_band;
};

__device__ __forceinline__ float epi_key(float r, int abs_mode) { return abs_mode ? fabsf(r) : r; }

__device__ __forceinline__ int epi_bin(float key, const EpiParams& p)
{
    float x = (key - p.kmin) * p.scale;
    int b = (int)x;
    if (!(x >= 0.0f)) b = 0;
    if (b > HIST_BINS - 1) b = HIST_BINS - 1;
    return b;
}

// Classification of one pair for EMIT: 0 = drop, 1 = decided edge, 2 = band.
__device__ __forceinline__ int epi_class(float r, const EpiParams& p)
{
    if (fabsf(r) >= p.edge_band) return 2;
    float k = epi_key(r, p.abs_mode);
    if (k >= p.hi_cut) return 1;
    if (k >= p.lo_cut) return 2;
    return 0;
}

// Appends for one (i, j, r) candidate; all lanes of the warp must call it.
__device__ __forceinline__ void epi_emit(int cls, int i, int j, float r, const EpiParams& p)
{
    long long s = warp_append(p.n_pairs, cls == 1);
    if (s >= 0 && s < p.cap_pairs) {
        p.pairs[s] = make_int2(i, j);
        if (p.weighted) p.pair_w[s] = epi_key(r, p.abs_mode);
    }
    long long b = warp_append(p.n_band, cls == 2);
    if (b >= 0 && b < p.cap_band) p.band[b] = make_int2(i, j);
}

// Upper-triangle tile enumeration: linear index L in [0, nb(nb+1)/2) ->
// (bi, bj) with bi <= bj, row-major.
__device__ __forceinline__ void tri_tile(long long L, int nb, int& bi, int& bj)
{
    long long nt = (long long)nb * (nb + 1) / 2;
    long long Lr = nt - 1 - L;
    long long r = (long long)((sqrt(8.0 * (double)Lr + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= Lr) r++;
    while (r * (r + 1) / 2 > Lr) r--;
    bi = nb - 1 - (int)r;
    bj = nb - 1 - (int)(Lr - r * (r + 1) / 2);
}

// Kernel launchers (defined in gram_simt.cu / gram_tc.cu).
pg_status launch_gram_simt(pg_ctx* ctx, const ZOperands& z, int mode, const EpiParams& p);
pg_status launch_gram_tc(pg_ctx* ctx, const ZOperands& z, int mode, const EpiParams& p);
bool gram_tc_supported(pg_ctx* ctx, const ZOperands& z);
