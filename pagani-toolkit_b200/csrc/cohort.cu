// cohort.cu -- subject-averaged correlation graphs: the to_average modes of
// CUCorMat (yn / yf / bn / bf; U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:380-620,
// W/CorMat/CUCorMat/CUCorMat/CorMat.cpp:386-620).
//
// The reference adds every subject's float r (or fisher_trans(r)) into a
// host array of M1 floats (post_block, CorMat.cpp:775-838), divides by the
// subject count, applies inv_fisher_trans (:514-524) and thresholds once.
// Here:
//   - one FP64 accumulator stays in HBM for the whole cohort, tile-major:
//     the 128 x 128 blocks (bi <= bj) of the pair matrix in row-major block
//     order, each block contiguous (13.5 GB at 58,000 voxels; positions with
//     j <= i or beyond N stay 0);
//   - per subject, FP64 z-scores are written time-major (T x Np, the layout
//     of the input series), then k_cohort_gram, a persistent FP64 Gram:
//     thread 0 streams 16 time points x 128 voxels of both operands per
//     stage with TMA into a 3-stage shared-memory ring (mbarrier waits
//     bounded by the global timer), every thread keeps an 8 x 8 block of
//     pair sums in registers -- one fused multiply-add per time point, t
//     ascending, the oracle's order -- and the epilogue applies the range
//     rule and the Fisher transform into a 128 KB shared-memory tile that
//     one asynchronous bulk reduce-add (cp.reduce.async.bulk .add.f64) adds
//     into the accumulator block while the next tile computes.  One add per
//     element and launch, so the sum is the oracle's, in subject order.  The tensor cores are not used: the average needs every
//     pair's exact FP64 r (no threshold separates decided pairs before all
//     subjects are summed) and tcgen05 has no FP64 kind;
//   - the graph: keys = order-preserving uint64 of acc / S (inverse Fisher
//     applied), then r mode counts and emits key > value, sparsity mode
//     selects the k-th key exactly (radix selection) with the reference's
//     tie rule, then the CSR is assembled.
// ln and exp are built from +, -, *, / in the oracle's order (Cody & Waite
// argument reduction and Taylor series), so keys, edges and weights are
// bit-identical to the oracle's.
#include "build_graph.cuh"
#include "tma.cuh"
#include <cuda.h>
#include <cstring>
#include <algorithm>

struct pg_cohort {
    int device = 0;
    int N = 0;
    int nb = 0;                            // 128-voxel blocks
    long long ntiles = 0;                  // nb (nb + 1) / 2 upper-triangle blocks
    long long nelem = 0;                   // ntiles * 128 * 128 accumulator entries
    int fisher = 0;
    int weighted = 0;
    int subjects = 0;
    long long M1 = 0;
    double* acc = nullptr;                 // device, nelem doubles (tile-major)
    unsigned long long* keys = nullptr;    // device, nelem keys, 0 where no pair (allocated on first use)
    bool keys_valid = false;
    bool broken = false;                   // an add failed part-way: the sums are unusable
};

namespace {
using namespace pg_tma;

// ------------------------------------------------------- FP64 ln and exp
// Method and constants as the oracle's or_ln / or_exp: ln x = e ln2 +
// 2 atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)), odd series to
// s^23; exp x = 2^k e^t, k = x/ln2 rounded half away from zero,
// t = (x - k ln2_hi) - k ln2_lo, Taylor series to t^14.  ln2_hi has 42
// significant bits (k ln2_hi exact for |k| < 2^11); coefficients 2/(2j+1)
// and 1/n! rounded to nearest.
constexpr double LN2_HI = 0x1.62e42fefa3800p-1, LN2_LO = 0x1.ef35793c76730p-45;
constexpr double INV_LN2 = 0x1.71547652b82fep+0, SQRT2 = 0x1.6a09e667f3bcdp+0;
__constant__ double c_atanh[11] = {
    0x1.5555555555555p-1, 0x1.999999999999ap-2, 0x1.2492492492492p-2, 0x1.c71c71c71c71cp-3,
    0x1.745d1745d1746p-3, 0x1.3b13b13b13b14p-3, 0x1.1111111111111p-3, 0x1.e1e1e1e1e1e1ep-4,
    0x1.af286bca1af28p-4, 0x1.8618618618618p-4, 0x1.642c8590b2164p-4};
__constant__ double c_exp[15] = {
    0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p-1, 0x1.5555555555555p-3,
    0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
    0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
    0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37};

__device__ __forceinline__ double neg_inf() { return __longlong_as_double(0xfff0000000000000LL); }
__device__ __forceinline__ double pos_inf() { return __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ double pow2i(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

__device__ double d_ln(double x)
{
    if (!(x >= 0.0)) return __longlong_as_double(0x7ff8000000000000LL);
    if (x == 0.0) return neg_inf();
    if (isinf(x)) return x;
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    int e = 0;
    if (((u >> 52) & 0x7ff) == 0) {
        x = __dmul_rn(x, 0x1p54);
        u = (unsigned long long)__double_as_longlong(x);
        e = -54;
    }
    e += (int)((u >> 52) & 0x7ff) - 1023;
    u = (u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m = __longlong_as_double((long long)u);
    if (m > SQRT2) { m = __dmul_rn(m, 0.5); e += 1; }
    const double s = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
    const double s2 = __dmul_rn(s, s);
    double p = c_atanh[10];
#pragma unroll
    for (int j = 9; j >= 0; j--) p = __dadd_rn(c_atanh[j], __dmul_rn(s2, p));
    const double ls = __dadd_rn(__dmul_rn(2.0, s), __dmul_rn(s, __dmul_rn(s2, p)));
    const double de = (double)e;
    return __dadd_rn(__dmul_rn(de, LN2_HI), __dadd_rn(__dmul_rn(de, LN2_LO), ls));
}

__device__ double d_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return pos_inf();
    if (x < -745.2) return 0.0;
    const double kd = __dmul_rn(x, INV_LN2);
    const long long k = (long long)__dadd_rn(kd, kd >= 0.0 ? 0.5 : -0.5);
    const double dk = (double)k;
    const double t = __dsub_rn(__dsub_rn(x, __dmul_rn(dk, LN2_HI)), __dmul_rn(dk, LN2_LO));
    double p = c_exp[14];
#pragma unroll
    for (int n = 13; n >= 0; n--) p = __dadd_rn(c_exp[n], __dmul_rn(t, p));
    if (k > 1023) return __dmul_rn(__dmul_rn(p, pow2i(1023)), pow2i((int)k - 1023));
    if (k < -1022) return __dmul_rn(__dmul_rn(p, pow2i((int)k + 600)), pow2i(-600));
    return __dmul_rn(p, pow2i((int)k));
}

// fisher_trans (CorMat.cpp:35-41) in FP64: r >= 1 -> 1 - 1e-6, r <= -1 -> -inf.
__device__ __forceinline__ double d_fisher(double r)
{
    if (r >= 1.0) r = 1.0 - 1e-6;
    if (r <= -1.0) return neg_inf();
    return __dmul_rn(0.5, d_ln(__ddiv_rn(__dadd_rn(1.0, r), __dsub_rn(1.0, r))));
}

// inv_fisher_trans (CorMat.cpp:43-49).
__device__ __forceinline__ double d_inv_fisher(double z)
{
    const double e = d_exp(__dmul_rn(2.0, z));
    return __ddiv_rn(__dsub_rn(e, 1.0), __dadd_rn(e, 1.0));
}

// post_block's range rule (U CorMat.cpp:821, W :833 with ep = 1e-6).
__device__ __forceinline__ double range_rule(double r, int weighted)
{
    if (weighted) return (r > -1.0 - 1e-6 && r < 1.0 + 1e-6) ? r : 0.0;
    return (r >= -1.0 && r <= 1.0) ? r : 0.0;
}

constexpr int CB = 128;          // voxels per block edge
constexpr int CB2 = CB * CB;     // accumulator entries per block

// Linear index of the first block of block row bi (blocks bi <= bj, row-major).
__device__ __forceinline__ long long block_row_start(long long bi, long long nb) { return bi * nb - bi * (bi - 1) / 2; }

// Block (bi, bj) of linear index L, by binary search over the row starts.
__device__ __forceinline__ int2 block_of(long long L, int nb)
{
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (block_row_start(mid, nb) <= L) lo = mid;
        else hi = mid - 1;
    }
    return make_int2(lo, lo + (int)(L - block_row_start(lo, nb)));
}

// Accumulator position of pair (i, j), i < j.
__device__ __forceinline__ long long acc_pos(int i, int j, int nb)
{
    const int bi = i / CB, bj = j / CB;
    return (block_row_start(bi, nb) + (bj - bi)) * CB2 + (long long)(i % CB) * CB + (j % CB);
}

// ------------------------------------------------------------ z-scores
// zT[t * Np + i] = (x - mean_i) / s_i with the operations of k_zwrite (the
// oracle's z); zero for padding rows/columns and zero-variance voxels.
__global__ void k_cohort_z(const float* __restrict__ bold, int N, int T, int Np, int Tp,
                           const double* __restrict__ mu, const double* __restrict__ sd, double* __restrict__ zT)
{
    const long long total = (long long)Tp * Np;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(q / Np), i = (int)(q % Np);
        double z = 0.0;
        if (t < T && i < N && sd[i] > 0.0)
            z = __ddiv_rn(__dsub_rn((double)bold[(size_t)t * N + i], mu[i]), sd[i]);
        zT[q] = z;
    }
}

// ------------------------------------------------------------ FP64 Gram
constexpr int CK = 16;           // time points per stage
constexpr int CSTAGES = 3;
constexpr int CTHREADS = 256;    // 16 x 16 threads, 8 x 8 pairs each
constexpr uint32_t CTILE_BYTES = CB * CK * 8;
constexpr uint32_t CSTAGE_BYTES = 2 * CTILE_BYTES;
constexpr uint32_t COUT_BYTES = CB2 * 8;            // 128 KB epilogue tile
constexpr size_t CSMEM = 128 + CSTAGES * CSTAGE_BYTES + COUT_BYTES + CSTAGES * 8 + 16;

struct CohortArgs {
    int N, T, nb, nk;
    long long ntiles;
    double* acc;
    int weighted;
    int* err;
};

// Block cursor over the row-major upper triangle of nb x nb blocks: block
// (bi, bi + rem).  Advances by `step` linear positions.
__device__ __forceinline__ void tile_advance(int nb, int& bi, long long& rem, long long step)
{
    rem += step;
    while (bi < nb && rem >= nb - bi) {
        rem -= nb - bi;
        bi++;
    }
}

__device__ __forceinline__ void bulk_reduce_add_f64(double* gdst, const void* ssrc, uint32_t bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;"
                 ::"l"(gdst), "r"(smem_u32(ssrc)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

template <bool FISHER>
__global__ void __launch_bounds__(CTHREADS, 1)
k_cohort_gram(const __grid_constant__ CUtensorMap zmap, const CohortArgs a)
{
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
    double* out = (double*)(sm + CSTAGES * CSTAGE_BYTES);
    unsigned long long* full = (unsigned long long*)(sm + CSTAGES * CSTAGE_BYTES + COUT_BYTES);
    volatile int* abort_flag = (volatile int*)(full + CSTAGES);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const long long G = gridDim.x;
    if ((long long)blockIdx.x >= a.ntiles) return;
    const long long total = ((a.ntiles - 1 - blockIdx.x) / G + 1) * a.nk;
    if (tid == 0) {
        for (int s = 0; s < CSTAGES; s++) mbar_init(&full[s], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // producer state (thread 0): block of the next chunk to issue
    int pbi = 0;
    long long prem = 0;
    tile_advance(a.nb, pbi, prem, blockIdx.x);
    auto issue = [&](long long q) {
        const int kc = (int)(q % a.nk);
        if (kc == 0 && q > 0) tile_advance(a.nb, pbi, prem, G);
        const int s = (int)(q % CSTAGES);
        unsigned char* base = sm + s * CSTAGE_BYTES;
        mbar_expect_tx(&full[s], CSTAGE_BYTES);
        tma_load(base, &zmap, pbi * CB, kc * CK, &full[s]);
        tma_load(base + CTILE_BYTES, &zmap, (int)(pbi + prem) * CB, kc * CK, &full[s]);
    };
    if (tid == 0)
        for (long long q = 0; q < total && q < CSTAGES; q++) issue(q);

    int cbi = 0;
    long long crem = 0, cL = blockIdx.x;
    tile_advance(a.nb, cbi, crem, blockIdx.x);
    double c[8][8];
    long long q = 0;
    for (; q < total; q++) {
        const int kc = (int)(q % a.nk);
        if (kc == 0) {
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int v = 0; v < 8; v++) c[u][v] = 0.0;
        }
        const int s = (int)(q % CSTAGES);
        if (!mbar_wait(&full[s], (uint32_t)((q / CSTAGES) & 1))) *abort_flag = 1;
        const double* A = (const double*)(sm + s * CSTAGE_BYTES);
        const double* B = A + CB * CK;
        const int kt = min(CK, a.T - kc * CK);
#pragma unroll 1
        for (int t = 0; t < kt; t++) {
            const double2* a2 = (const double2*)(A + t * CB);
            const double2* b2 = (const double2*)(B + t * CB);
            double ra[8], rb[8];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double2 x = a2[ty + 16 * u];
                const double2 y = b2[tx + 16 * u];
                ra[2 * u] = x.x;
                ra[2 * u + 1] = x.y;
                rb[2 * u] = y.x;
                rb[2 * u + 1] = y.y;
            }
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int v = 0; v < 8; v++) c[u][v] = __fma_rn(ra[u], rb[v], c[u][v]);
        }
        if (kc == a.nk - 1 && tid == 0)
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");   // the last block's reduce has read `out`
        __syncthreads();                       // every thread is done with stage s (and `out` is free)
        if (*abort_flag) break;
        if (tid == 0 && q + CSTAGES < total) issue(q + CSTAGES);
        if (kc == a.nk - 1) {
            const int I0 = cbi * CB, J0 = (int)(cbi + crem) * CB;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int r = 2 * ty + 32 * (u >> 1) + (u & 1);
                const int i = I0 + r;
#pragma unroll
                for (int v = 0; v < 8; v += 2) {
                    const int cl = 2 * tx + 32 * (v >> 1);
                    double2 f;
                    f.x = f.y = 0.0;
                    const int j = J0 + cl;
                    if (j > i && j < a.N) {
                        const double x = range_rule(c[u][v], a.weighted);
                        f.x = FISHER ? d_fisher(x) : x;
                    }
                    if (j + 1 > i && j + 1 < a.N) {
                        const double x = range_rule(c[u][v + 1], a.weighted);
                        f.y = FISHER ? d_fisher(x) : x;
                    }
                    *(double2*)(out + r * CB + cl) = f;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // `out` visible to the bulk copy
            __syncthreads();
            if (tid == 0) bulk_reduce_add_f64(a.acc + cL * CB2, out, COUT_BYTES);
            tile_advance(a.nb, cbi, crem, G);
            cL += G;
        }
    }
    if (tid == 0) {
        if (q < total) {
            // a wait timed out: record it and drain this CTA's loads in flight
            atomicExch(a.err, 1);
            const long long last = total < q + CSTAGES ? total : q + CSTAGES;
            for (long long w = q; w < last; w++)
                mbar_wait(&full[w % CSTAGES], (uint32_t)((w / CSTAGES) & 1), WAIT_NS / 4);
        }
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");   // reduces complete before exit
    }
}

// ------------------------------------------------------ keys and graph
// Kernels over the accumulator run one block of 256 threads per 128 x 128
// accumulator block (grid-stride over blocks).

template <bool FISHER>
__global__ void k_cohort_keys(const double* __restrict__ acc, int N, int nb, long long ntiles, double subjects,
                              unsigned long long* __restrict__ keys)
{
    for (long long L = blockIdx.x; L < ntiles; L += gridDim.x) {
        const int2 b = block_of(L, nb);
        const double* src = acc + L * CB2;
        unsigned long long* dst = keys + L * CB2;
        for (int e = threadIdx.x; e < CB2; e += blockDim.x) {
            const int i = b.x * CB + (e >> 7), j = b.y * CB + (e & 127);
            unsigned long long k = 0;
            if (j > i && j < N) {
                double x = __ddiv_rn(src[e], subjects);
                if (FISHER) x = d_inv_fisher(x);
                k = dkey(x);
            }
            dst[e] = k;
        }
    }
}

// CMP 0 counts keys > tkey, CMP 1 keys == tkey (tkey > 0: the 0 of an empty
// position never counts).
template <int CMP>
__global__ void k_cohort_count(const unsigned long long* __restrict__ keys, long long n, unsigned long long tkey,
                               unsigned long long* __restrict__ count)
{
    unsigned long long local = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[p];
        local += CMP == 0 ? (k > tkey) : (k == tkey);
    }
    for (int o = 16; o; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// Complemented lexicographic keys ~(i*N + j) of the pairs tied at tkey, so
// that selecting the m-th largest yields the m-th smallest pair.
__global__ void k_cohort_tie_keys(const unsigned long long* __restrict__ keys, int N, int nb, long long ntiles,
                                  unsigned long long tkey, unsigned long long* __restrict__ out,
                                  unsigned long long* __restrict__ n, long long cap)
{
    for (long long L = blockIdx.x; L < ntiles; L += gridDim.x) {
        const int2 b = block_of(L, nb);
        for (int e = threadIdx.x; e < CB2; e += blockDim.x) {
            const bool in = keys[L * CB2 + e] == tkey;
            const long long s = warp_append(n, in);
            if (s >= 0 && s < cap) {
                const unsigned long long i = b.x * CB + (e >> 7), j = b.y * CB + (e & 127);
                out[s] = ~(i * (unsigned long long)N + j);
            }
        }
    }
}

// Edges: key > tkey, or key == tkey and (i, j) <= tie_cut lexicographically.
__global__ void k_cohort_emit(const unsigned long long* __restrict__ keys, int N, int nb, long long ntiles,
                              unsigned long long tkey, int strict_only, unsigned long long tie_cut, int weighted,
                              int2* __restrict__ pairs, float* __restrict__ w, unsigned long long* __restrict__ n,
                              long long cap)
{
    for (long long L = blockIdx.x; L < ntiles; L += gridDim.x) {
        const int2 b = block_of(L, nb);
        for (int e = threadIdx.x; e < CB2; e += blockDim.x) {
            const unsigned long long k = keys[L * CB2 + e];
            const int i = b.x * CB + (e >> 7), j = b.y * CB + (e & 127);
            const bool in = k > tkey || (!strict_only && k == tkey &&
                                         (unsigned long long)i * (unsigned long long)N + (unsigned long long)j <= tie_cut);
            const long long s = warp_append(n, in);
            if (s >= 0 && s < cap) {
                pairs[s] = make_int2(i, j);
                if (weighted) w[s] = (float)dkey_inv(k);
            }
        }
    }
}

// Packed upper triangle (the .cormat order) of rows [row0, row0 + rows):
// one warp per row, lanes over j.
__global__ void k_cohort_packed(const unsigned long long* __restrict__ keys, int N, int nb, long long row0,
                                long long rows, float* __restrict__ out)
{
    const long long base0 = row0 * N - row0 * (row0 + 1) / 2;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (long long ii = warp; ii < rows; ii += nw) {
        const int i = (int)(row0 + ii);
        const long long off = (long long)i * N - (long long)i * (i + 1) / 2 - base0;
        for (int j = i + 1 + lane; j < N; j += 32) out[off + (j - i - 1)] = (float)dkey_inv(keys[acc_pos(i, j, nb)]);
    }
}

bool make_zmap(CUtensorMap* m, const double* base, int Np, int Tp)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Np, (cuuint64_t)Tp};
    cuuint64_t strides[1] = {(cuuint64_t)Np * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)CB, (cuuint32_t)CK};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void*)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

pg_status check_cohort(pg_ctx* ctx, const pg_cohort* c, const char* fn)
{
    if (!ctx || !c) return pg_fail(ctx, PG_ERR_INVALID, "%s: null argument", fn);
    if (c->device != ctx->device)
        return pg_fail(ctx, PG_ERR_INVALID, "%s: cohort lives on device %d, context on %d", fn, c->device, ctx->device);
    if (c->broken) return pg_fail(ctx, PG_ERR_INVALID, "%s: an earlier add failed; the cohort is unusable", fn);
    return PG_OK;
}

int block_grid(pg_ctx* ctx, long long ntiles) { return (int)std::max(1LL, std::min<long long>(ctx->sm_count * 8LL, ntiles)); }

// keys = dkey(finish(acc)) (0 where there is no pair), computed once after
// the last add.
pg_status cohort_keys(pg_ctx* ctx, pg_cohort* c)
{
    if (c->subjects < 1) return pg_fail(ctx, PG_ERR_INVALID, "cohort has no subjects");
    if (c->keys_valid) return PG_OK;
    if (!c->keys) PG_CUDA(ctx, cudaMalloc(&c->keys, sizeof(unsigned long long) * (size_t)c->nelem));
    const int grid = block_grid(ctx, c->ntiles);
    if (c->fisher)
        k_cohort_keys<true><<<grid, 256, 0, ctx->stream>>>(c->acc, c->N, c->nb, c->ntiles, (double)c->subjects, c->keys);
    else
        k_cohort_keys<false><<<grid, 256, 0, ctx->stream>>>(c->acc, c->N, c->nb, c->ntiles, (double)c->subjects, c->keys);
    PG_LAUNCHED(ctx);
    c->keys_valid = true;
    return PG_OK;
}
}  // namespace

// ------------------------------------------------------------------ API
extern "C" pg_status pg_cohort_create(pg_ctx* ctx, int32_t N, int32_t fisher, int32_t weighted, pg_cohort** out)
{
    if (!ctx || !out || N < 1) return pg_fail(ctx, PG_ERR_INVALID, "pg_cohort_create: bad arguments (N=%d)", N);
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->smem_optin < CSMEM)
        return pg_fail(ctx, PG_ERR_CUDA, "pg_cohort_create: %zu B of shared memory per block needed, %zu available",
                       CSMEM, ctx->smem_optin);
    *out = nullptr;
    pg_cohort* c = new pg_cohort;
    c->device = ctx->device;
    c->N = N;
    c->nb = (N + CB - 1) / CB;
    c->ntiles = (long long)c->nb * (c->nb + 1) / 2;
    c->nelem = c->ntiles * CB2;
    c->fisher = fisher != 0;
    c->weighted = weighted != 0;
    c->M1 = (long long)N * (N - 1) / 2;
    cudaError_t e = cudaMalloc(&c->acc, sizeof(double) * (size_t)c->nelem);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->acc, 0, sizeof(double) * (size_t)c->nelem, ctx->stream);
    if (e != cudaSuccess) {
        const long long nelem = c->nelem;
        pg_cohort_free(c);
        return pg_fail(ctx, e == cudaErrorMemoryAllocation ? PG_ERR_NOMEM : PG_ERR_CUDA,
                       "pg_cohort_create: %lld-entry accumulator: %s", nelem, cudaGetErrorString(e));
    }
    *out = c;
    return PG_OK;
}

extern "C" pg_status pg_cohort_add(pg_ctx* ctx, pg_cohort* c, const float* bold, int32_t T, int32_t input_on_device)
{
    PG_TRY(check_cohort(ctx, c, "pg_cohort_add"));
    if (!bold || T < 1) return pg_fail(ctx, PG_ERR_INVALID, "pg_cohort_add: bad arguments (T=%d)", T);
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int N = c->N, Np = c->nb * CB, Tp = (T + CK - 1) / CK * CK;
    const float* dbold = bold;
    if (!input_on_device) {
        float* tmp;
        PG_TRY(pg_wst(ctx, "bold", (size_t)N * T, &tmp));
        PG_CUDA(ctx, cudaMemcpyAsync(tmp, bold, sizeof(float) * (size_t)N * T, cudaMemcpyHostToDevice, ctx->stream));
        dbold = tmp;
    }
    double *mu, *sd, *zT;
    int *nz, *err;
    PG_TRY(pg_wst(ctx, "z.mu", (size_t)N, &mu));
    PG_TRY(pg_wst(ctx, "z.sd", (size_t)N, &sd));
    PG_TRY(pg_wst(ctx, "z.nzero", 1, &nz));
    PG_TRY(pg_wst(ctx, "cohort.zT", (size_t)Np * Tp, &zT));
    PG_TRY(pg_wst(ctx, "cohort.err", 1, &err));
    PG_TRY(pg_zstats(ctx, dbold, N, T, mu, sd, nz));
    {
        const int grid = std::max(1, std::min(ctx->sm_count * 8, ceil_div((long long)Np * Tp, 256)));
        k_cohort_z<<<grid, 256, 0, ctx->stream>>>(dbold, N, T, Np, Tp, mu, sd, zT);
        PG_LAUNCHED(ctx);
    }
    c->keys_valid = false;
    c->subjects++;
    if (c->M1 == 0) return PG_OK;
    CUtensorMap zmap;
    if (!make_zmap(&zmap, zT, Np, Tp))
        return pg_fail(ctx, PG_ERR_CUDA, "cuTensorMapEncodeTiled failed for the cohort z-scores");
    CohortArgs a;
    a.N = N;
    a.T = T;
    a.nb = c->nb;
    a.nk = Tp / CK;
    a.ntiles = c->ntiles;
    a.acc = c->acc;
    a.weighted = c->weighted;
    a.err = err;
    PG_CUDA(ctx, cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    const int grid = (int)std::min<long long>(ctx->sm_count, a.ntiles);
    if (c->fisher) {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_cohort_gram<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CSMEM));
        k_cohort_gram<true><<<grid, CTHREADS, CSMEM, ctx->stream>>>(zmap, a);
    } else {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_cohort_gram<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CSMEM));
        k_cohort_gram<false><<<grid, CTHREADS, CSMEM, ctx->stream>>>(zmap, a);
    }
    PG_LAUNCHED(ctx);
    int herr = 0;
    PG_TRY(pg_d2h(ctx, &herr, err, sizeof(int)));
    if (herr) {
        c->broken = true;   // the accumulator may hold part of this subject
        return pg_fail(ctx, PG_ERR_TIMEOUT, "cohort Gram: a pipeline wait timed out; the cohort is unusable");
    }
    return PG_OK;
}

extern "C" pg_status pg_cohort_graph(pg_ctx* ctx, pg_cohort* c, int32_t mode, double value, pg_graph** out,
                                     pg_build_info* info)
{
    PG_TRY(check_cohort(ctx, c, "pg_cohort_graph"));
    if (!out) return pg_fail(ctx, PG_ERR_INVALID, "pg_cohort_graph: null output");
    if (mode != PG_THRESH_R && mode != PG_THRESH_SPARSITY)
        return pg_fail(ctx, PG_ERR_INVALID, "unknown threshold mode %d", mode);
    if (mode == PG_THRESH_SPARSITY && (!(value >= 0.0) || value > 100.0))
        return pg_fail(ctx, PG_ERR_INVALID, "sparsity %g%% out of range", value);
    if (mode == PG_THRESH_R && value != value) return pg_fail(ctx, PG_ERR_INVALID, "r threshold is NaN");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nullptr;
    pg_build_info inf;
    memset(&inf, 0, sizeof inf);
    cudaEvent_t* ev = ctx->ev;
    PG_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));
    PG_TRY(cohort_keys(ctx, c));
    PG_CUDA(ctx, cudaEventRecord(ev[1], ctx->stream));
    const int N = c->N;
    const long long M1 = c->M1;
    const int egrid = std::max(1, std::min(ctx->sm_count * 8, ceil_div(c->nelem, 256)));
    const int bgrid = block_grid(ctx, c->ntiles);
    unsigned long long* counters;
    PG_TRY(pg_wst(ctx, "cohort.counters", 4, &counters));
    PG_CUDA(ctx, cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), ctx->stream));
    unsigned long long tkey = 0, tie_cut = 0;
    int strict_only = 1;
    long long n_edges = 0;
    double tau = value;
    if (mode == PG_THRESH_R) {
        tau = value + 0.0;   // -0 threshold behaves as +0 (keys are never -0)
        tkey = dkey(tau);
        k_cohort_count<0><<<egrid, 256, 0, ctx->stream>>>(c->keys, c->nelem, tkey, counters);
        PG_LAUNCHED(ctx);
        unsigned long long nh = 0;
        PG_TRY(pg_d2h(ctx, &nh, counters, sizeof nh));
        n_edges = (long long)nh;
    } else {
        long long k_edges = pg_sparsity_edges(N, (float)value);
        if (k_edges > M1) k_edges = M1;
        if (k_edges <= 0) {
            tau = INFINITY;
            tkey = ~0ULL;
        } else {
            SelState* st;
            unsigned long long* hist;
            PG_TRY(pg_wst(ctx, "cohort.sel", 2, &st));
            PG_TRY(pg_wst(ctx, "cohort.hist", 256, &hist));
            PG_TRY(pg_radix_select(ctx, c->keys, c->nelem, k_edges, st, hist));
            SelState sh;
            PG_TRY(pg_d2h(ctx, &sh, st, sizeof sh));
            tkey = sh.prefix;
            tau = dkey_inv(tkey);
            const long long need = sh.m;   // ties at tau still to take (>= 1)
            k_cohort_count<1><<<egrid, 256, 0, ctx->stream>>>(c->keys, c->nelem, tkey, counters + 1);
            PG_LAUNCHED(ctx);
            unsigned long long nt = 0;
            PG_TRY(pg_d2h(ctx, &nt, counters + 1, sizeof nt));
            strict_only = 0;
            if ((long long)nt <= need) {
                tie_cut = ~0ULL;
            } else {
                unsigned long long* tk;
                PG_TRY(pg_wst(ctx, "cohort.ties", (size_t)nt, &tk));
                k_cohort_tie_keys<<<bgrid, 256, 0, ctx->stream>>>(c->keys, N, c->nb, c->ntiles, tkey, tk, counters + 2,
                                                                  (long long)nt);
                PG_LAUNCHED(ctx);
                PG_TRY(pg_radix_select(ctx, tk, (long long)nt, need, st, hist));
                PG_TRY(pg_d2h(ctx, &sh, st, sizeof sh));
                tie_cut = ~sh.prefix;
            }
        }
        n_edges = k_edges > 0 ? k_edges : 0;
    }
    PG_CUDA(ctx, cudaEventRecord(ev[2], ctx->stream));
    if (n_edges > (long long)INT32_MAX) return pg_fail(ctx, PG_ERR_TOO_LARGE, "too many edges (%lld)", n_edges);
    int2* pairs;
    float* pw = nullptr;
    PG_TRY(pg_wst(ctx, "b.pairs", (size_t)std::max(1LL, n_edges), &pairs));
    if (c->weighted) PG_TRY(pg_wst(ctx, "b.pw", (size_t)std::max(1LL, n_edges), &pw));
    if (n_edges > 0) {
        k_cohort_emit<<<bgrid, 256, 0, ctx->stream>>>(c->keys, N, c->nb, c->ntiles, tkey, strict_only, tie_cut,
                                                      c->weighted, pairs, pw, counters + 3, n_edges);
        PG_LAUNCHED(ctx);
        unsigned long long ne = 0;
        PG_TRY(pg_d2h(ctx, &ne, counters + 3, sizeof ne));
        if ((long long)ne != n_edges)
            return pg_fail(ctx, PG_ERR_INTERNAL, "cohort graph has %llu edges, expected %lld", ne, n_edges);
    }
    pg_graph* g;
    PG_TRY(pg_csr_from_pairs(ctx, N, pairs, pw, n_edges, &g));
    cudaError_t e = cudaEventRecord(ev[3], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        pg_graph_free(g);
        return pg_fail(ctx, PG_ERR_CUDA, "pg_cohort_graph: %s", cudaGetErrorString(e));
    }
    float ms;
    cudaEventElapsedTime(&ms, ev[0], ev[1]); inf.ms_zscore = ms;   // keys (finish of the average)
    cudaEventElapsedTime(&ms, ev[1], ev[2]); inf.ms_select = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]); inf.ms_csr = ms;
    inf.tau = tau;
    inf.edges = n_edges;
    inf.sparsity_percent = M1 > 0 ? 100.0 * (double)n_edges / (double)M1 : 0.0;
    if (info) *info = inf;
    *out = g;
    return PG_OK;
}

extern "C" pg_status pg_cohort_packed(pg_ctx* ctx, pg_cohort* c, float* r_packed)
{
    PG_TRY(check_cohort(ctx, c, "pg_cohort_packed"));
    if (!r_packed) return pg_fail(ctx, PG_ERR_INVALID, "pg_cohort_packed: null output");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    PG_TRY(cohort_keys(ctx, c));
    const int N = c->N;
    const long long chunk_elems = 64LL << 20;
    float* buf;
    PG_TRY(pg_wst(ctx, "cormat.out", (size_t)std::min(std::max(c->M1, 1LL), chunk_elems + N), &buf));
    long long row = 0;
    while (row < N - 1) {
        long long r1 = row, elems = 0;
        while (r1 < N - 1 && elems + (N - 1 - r1) <= std::max(chunk_elems, (long long)N)) {
            elems += N - 1 - r1;
            r1++;
        }
        const long long off = row * N - row * (row + 1) / 2;
        k_cohort_packed<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(c->keys, N, c->nb, row, r1 - row, buf);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_d2h(ctx, r_packed + off, buf, sizeof(float) * (size_t)elems));
        row = r1;
    }
    return PG_OK;
}

extern "C" pg_status pg_cohort_info(const pg_cohort* c, int32_t* N, int32_t* subjects)
{
    if (!c) return PG_ERR_INVALID;
    if (N) *N = c->N;
    if (subjects) *subjects = c->subjects;
    return PG_OK;
}

extern "C" pg_status pg_cohort_free(pg_cohort* c)
{
    if (!c) return PG_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(c->device);
    if (c->acc) cudaFree(c->acc);
    if (c->keys) cudaFree(c->keys);
    cudaSetDevice(cur);
    delete c;
    return PG_OK;
}
