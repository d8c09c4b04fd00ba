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
    int tile_stride;               // HIST: visit every tile_stride-th tile only (sampling)
    // HIST: keys below kmin are only counted; the rest go to
    // bin = clamp((key - kmin) * scale)
    float kmin, scale;
    unsigned int* hist;            // HIST_BINS global counters
    unsigned long long* below;     // [0] keys < kmin, [1] pairs with r <= -edge_band
    // EMIT: key >= hi_cut -> decided edge; key >= lo_cut -> FP64 band;
    // |r| >= edge_band -> band (range rule near +-1).
    float lo_cut, hi_cut, edge_band;
    int2* pairs;                   // decided edges (i < j)
    float* pair_w;                 // their weights (weighted only)
    unsigned long long* n_pairs;
    long long cap_pairs;
    int2* band;                    // band pairs (i < j)
    float* band_r;                 // the tile's r of every band pair
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

// HIST for one valid pair: count below the floor in registers, bin the rest
// in the shared-memory histogram.
__device__ __forceinline__ void epi_hist(float r, const EpiParams& p, unsigned int* sh_hist,
                                         unsigned int& below, unsigned int& neg)
{
    float k = epi_key(r, p.abs_mode);
    neg += (!p.abs_mode && r <= -p.edge_band);
    if (k < p.kmin) below++;
    else atomicAdd(&sh_hist[epi_bin(k, p)], 1u);
}

// Flush the per-thread HIST counters: one atomic per warp.
__device__ __forceinline__ void epi_hist_flush(unsigned int below, unsigned int neg, const EpiParams& p)
{
    unsigned int b = __reduce_add_sync(0xffffffffu, below);
    unsigned int n = __reduce_add_sync(0xffffffffu, neg);
    if ((threadIdx.x & 31) == 0) {
        if (b) atomicAdd(&p.below[0], (unsigned long long)b);
        if (n) atomicAdd(&p.below[1], (unsigned long long)n);
    }
}

// Reserve c slots per lane in a global list with one atomic per warp; returns
// this lane's first slot.
__device__ __forceinline__ long long warp_reserve(unsigned long long* counter, unsigned int c)
{
    const int lane = threadIdx.x & 31;
    unsigned int x = c;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    unsigned int total = __shfl_sync(0xffffffffu, x, 31);
    unsigned long long base = 0;
    if (lane == 31 && total) base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    return (long long)(base + (x - c));
}

// EMIT for a run of up to 32 candidates per lane.  m1/m2 flag "decided edge"
// / "band" per candidate slot; (i, j, r) of slot q come from `at(q, i, j, r)`.
// The slot loop is unrolled so that `at` may index register arrays.
template <class At>
__device__ __forceinline__ void epi_emit_masks(unsigned int m1, unsigned int m2, const EpiParams& p, At at)
{
    if (!__any_sync(0xffffffffu, (m1 | m2) != 0u)) return;
    long long s1 = warp_reserve(p.n_pairs, __popc(m1));
    long long s2 = warp_reserve(p.n_band, __popc(m2));
    if (!(m1 | m2)) return;
#pragma unroll
    for (int q = 0; q < 32; q++) {
        const bool e1 = (m1 >> q) & 1u, e2 = (m2 >> q) & 1u;
        if (e1 | e2) {
            int i, j;
            float r;
            at(q, i, j, r);
            if (e1) {
                if (s1 < p.cap_pairs) {
                    p.pairs[s1] = make_int2(i, j);
                    if (p.weighted) p.pair_w[s1] = epi_key(r, p.abs_mode);
                }
                s1++;
            } else {
                if (s2 < p.cap_band) {
                    p.band[s2] = make_int2(i, j);
                    p.band_r[s2] = r;
                }
                s2++;
            }
        }
    }
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

// Radix selection state (device): the m-th largest of n uint64 keys is found
// 8 bits per pass from the top; `prefix` holds its bits when done.
struct SelState {
    unsigned long long prefix, mask;
    long long m;         // rank still to find inside the current prefix
    long long above;     // number of keys strictly above the final key
};
// m-th largest (1-based) of n keys; hist is 256 device counters.
pg_status pg_radix_select(pg_ctx* ctx, const unsigned long long* keys, long long n, long long m,
                          SelState* st_dev, unsigned long long* hist);
// FP64 z-score statistics of a device T x N series (k_zstats): mean and root
// sum of squares per voxel, sd = 0 for zero-variance voxels, counted in *nz.
pg_status pg_zstats(pg_ctx* ctx, const float* dbold, int N, int T, double* mu, double* sd, int* nz);
