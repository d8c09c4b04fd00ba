// eigen.cu -- eigenvector centrality by the power method of the CUEC tools
// (Lead_Vector_GPU, U/CUEC/CUEC/CUEC_unweighted.cu:61-214 and
// W/CUEC/weighted-net.cu:55-218).
//
// The reference step is u0 = u; vNorm = |u|; u = u * (1/vNorm); y = A u;
// err1 = |y - u0|, err2 = |y + u0|, with u starting as the node ids; it stops
// when err1 or err2 is at most 1e-6 or after 10,000 steps.  Here the whole
// iteration is one cooperative launch over the GPU.  Each CTA owns an
// edge-balanced range of rows; a step walks the vector in column blocks of
// 2^cb_log entries that every CTA copies into shared memory, scaled by
// 1/vNorm on the way in (the reference's normalised u), and adds the block's
// share of each own row.  Columns are read as 16-bit offsets inside their
// block (a copy made at the start of the launch).  The three sums of a step
// -- |y - u0|^2, |y + u0|^2 and |y|^2 (the next step's vNorm) -- meet in one
// grid-wide reduction, in the same fixed order in every block.
#include "pg_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>

namespace cg = cooperative_groups;

namespace {
constexpr int EC_THREADS = 1024;
constexpr int EC_MAX_ITER = 10000;
constexpr double EC_EPSILON = 1e-6;

struct EcArgs {
    const int32_t* R;
    const int32_t* C;
    const float* V;        // null: every edge counts 1
    int n;
    int cb_log;            // column block = 2^cb_log entries
    double* u0;            // unnormalised vectors of alternate steps
    double* u1;
    double* part;          // [2][gridDim.x][4] block sums, alternate halves
    uint16_t* c16;         // columns modulo the block size
    double* x_out;         // normalised vector of the last step
    double* y_out;         // y = A x of the last step
    double* info;          // eigenvalue, steps, residual
    double err_sq;         // largest double whose square root is at most 1e-6
};

// first row whose edge offset reaches rank * nnz / nb
__host__ __device__ inline int ec_split(const int32_t* R, int n, int rank, int nb)
{
    if (rank <= 0) return 0;
    if (rank >= nb) return n;
    const long long target = (long long)R[n] * rank / nb;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (R[mid] >= target) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__host__ __device__ inline size_t ec_smem(int nown, int nblk, int cb)
{
    return (size_t)cb * 8 + (size_t)nown * 8 + ((size_t)(nblk + 1) * nown * 4 + 15) / 16 * 16;
}

__device__ __forceinline__ void warp_sum3(double* x)
{
#pragma unroll
    for (int q = 0; q < 3; q++)
        for (int o = 16; o; o >>= 1) x[q] += __shfl_xor_sync(0xffffffffu, x[q], o);
}

// sums of three values over the grid; every block folds the block values in
// the same order, so all threads end with bit-identical sums
struct GridSum3 {
    double warp[2][32][3];
    double bc[2][3];
    __device__ void sum(double* x, int& ph, double* part)
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        warp_sum3(x);
        if (lane == 0)
            for (int q = 0; q < 3; q++) warp[ph][w][q] = x[q];
        __syncthreads();
        double* pp = part + (size_t)ph * gridDim.x * 4;
        if (w == 0) {
            for (int q = 0; q < 3; q++) x[q] = lane < nw ? warp[ph][lane][q] : 0.0;
            warp_sum3(x);
            if (lane < 3) pp[blockIdx.x * 4 + lane] = lane == 0 ? x[0] : lane == 1 ? x[1] : x[2];
        }
        // the other half of `part` is written next, this one again only
        // after another grid barrier
        cg::this_grid().sync();
        if (w == 0) {
            x[0] = x[1] = x[2] = 0.0;
            for (int b = lane; b < (int)gridDim.x; b += 32)
                for (int q = 0; q < 3; q++) x[q] += pp[b * 4 + q];
            warp_sum3(x);
            if (lane < 3) bc[ph][lane] = lane == 0 ? x[0] : lane == 1 ? x[1] : x[2];
        }
        __syncthreads();
        for (int q = 0; q < 3; q++) x[q] = bc[ph][q];
        ph ^= 1;
    }
};

// add column block b's share of every own row to ypart, L lanes per row
template <int L, bool W>
__device__ __forceinline__ void ec_rows(const EcArgs& a, const double* vb, const int32_t* split, int nblk, int nown,
                                        double* ypart, int b, int lane, int wid, int nwarp)
{
    constexpr int RPW = 32 / L;
    const int sub = lane & (L - 1);
    const uint16_t* __restrict__ cols = a.c16;
    for (int base = wid * RPW; base < nown; base += nwarp * RPW) {
        const int lp = base + lane / L;
        const bool act = lp < nown;
        int q = 0, q1 = 0;
        if (act) {
            q = split[lp * (nblk + 1) + b] + sub;
            q1 = split[lp * (nblk + 1) + b + 1];
        }
        double s0 = 0.0, s1 = 0.0;
        for (; q + L < q1; q += 2 * L) {
            if (W) {
                s0 = __dadd_rn(s0, __dmul_rn((double)a.V[q], vb[cols[q]]));
                s1 = __dadd_rn(s1, __dmul_rn((double)a.V[q + L], vb[cols[q + L]]));
            } else {
                s0 += vb[cols[q]];
                s1 += vb[cols[q + L]];
            }
        }
        if (q < q1) s0 = W ? __dadd_rn(s0, __dmul_rn((double)a.V[q], vb[cols[q]])) : s0 + vb[cols[q]];
        double y = s0 + s1;
        for (int o = L / 2; o; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (act && sub == 0) ypart[lp] = b == 0 ? y : ypart[lp] + y;
    }
}

template <bool W>
__device__ __forceinline__ void ec_block(int L, const EcArgs& a, const double* vb, const int32_t* split, int nblk,
                                         int nown, double* ypart, int b, int lane, int wid, int nwarp)
{
    switch (L) {
    case 1: ec_rows<1, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    case 2: ec_rows<2, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    case 4: ec_rows<4, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    case 8: ec_rows<8, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    case 16: ec_rows<16, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    default: ec_rows<32, W>(a, vb, split, nblk, nown, ypart, b, lane, wid, nwarp); return;
    }
}

// lanes per row: about 8 entries per lane, widened while rows alone leave
// threads idle
__device__ __forceinline__ int ec_lanes(int nown, long long entries, int nthr)
{
    const long long avg = nown > 0 ? entries / nown : 0;
    int L = 1;
    while (L < 32 && (long long)L * 8 <= avg) L <<= 1;
    while (L < 32 && (long long)nown * L < nthr && 2LL * L <= avg) L <<= 1;
    return L;
}

template <bool W>
__global__ void __launch_bounds__(EC_THREADS, 1) k_ec(EcArgs a)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ GridSum3 gs;
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, wid = tid >> 5, nwarp = nthr >> 5;
    const int n = a.n, cb = 1 << a.cb_log, nblk = (n + cb - 1) >> a.cb_log;
    const int r0 = ec_split(a.R, n, blockIdx.x, gridDim.x), r1 = ec_split(a.R, n, blockIdx.x + 1, gridDim.x);
    const int nown = r1 - r0;
    double* vblk = (double*)sm;
    double* ypart = vblk + cb;
    int32_t* split = (int32_t*)(ypart + nown);
    // own edges as 16-bit offsets in their column block; each own row's edge
    // range per block (columns ascend within a row)
    for (int q = a.R[r0] + tid; q < a.R[r1]; q += nthr) a.c16[q] = (uint16_t)(a.C[q] & (cb - 1));
    for (int lp = tid; lp < nown; lp += nthr) {
        const int p = r0 + lp, e0 = a.R[p], e1 = a.R[p + 1];
        int32_t* sp = split + lp * (nblk + 1);
        sp[0] = e0;
        for (int b = 1; b < nblk; b++) {
            int lo = e0, hi = e1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (a.C[mid] >= b * cb) hi = mid;
                else lo = mid + 1;
            }
            sp[b] = lo;
        }
        sp[nblk] = e1;
    }
    // u = node ids (init_AD); its norm is the first vNorm
    double x[3] = {0.0, 0.0, 0.0};
    for (int lp = tid; lp < nown; lp += nthr) {
        const double id = (double)(r0 + lp);
        a.u0[r0 + lp] = id;
        x[2] += id * id;
    }
    int ph = 0;
    gs.sum(x, ph, a.part);   // also publishes the start vector
    double vnorm = sqrt(x[2]), lam = 0.0;
    const int L = ec_lanes(nown, nown > 0 ? (long long)(a.R[r1] - a.R[r0]) / nblk : 0, nthr);
    double s1 = 1.0, s2 = 1.0;
    int iter = 0, cur = 0;
    while (s1 > a.err_sq && s2 > a.err_sq && iter < EC_MAX_ITER) {
        const double inv = 1.0 / vnorm;
        const double* uc = cur ? a.u1 : a.u0;
        double* un = cur ? a.u0 : a.u1;
        for (int b = 0; b < nblk; b++) {
            const int len = min(cb, n - b * cb);
            const double* src = uc + (size_t)b * cb;
            for (int p = tid; p < len; p += nthr) vblk[p] = src[p] * inv;
            __syncthreads();
            ec_block<W>(L, a, vblk, split, nblk, nown, ypart, b, lane, wid, nwarp);
            __syncthreads();
        }
        x[0] = x[1] = x[2] = 0.0;
        for (int lp = tid; lp < nown; lp += nthr) {
            const double y = ypart[lp], u0 = uc[r0 + lp];
            un[r0 + lp] = y;
            const double d1 = y - u0, d2 = y + u0;
            x[0] += d1 * d1;
            x[1] += d2 * d2;
            x[2] += y * y;
        }
        gs.sum(x, ph, a.part);   // also publishes y as the next u
        s1 = x[0];
        s2 = x[1];
        lam = vnorm;
        vnorm = sqrt(x[2]);
        cur ^= 1;
        iter++;
    }
    // last step: x = u * (1/vNorm) and y = A x, own rows
    const double inv = 1.0 / lam;
    const double* ul = cur ? a.u0 : a.u1;   // the last step's u
    const double* yl = cur ? a.u1 : a.u0;   // and its y
    for (int lp = tid; lp < nown; lp += nthr) {
        a.x_out[r0 + lp] = ul[r0 + lp] * inv;
        a.y_out[r0 + lp] = yl[r0 + lp];
    }
    if (blockIdx.x == 0 && tid == 0) {
        a.info[0] = lam;
        a.info[1] = iter;
        a.info[2] = fmin(sqrt(s1), sqrt(s2));
    }
}
}  // namespace

extern "C" pg_status pg_eigen_centrality(pg_ctx* ctx, const pg_graph* g, int32_t raw, double* ec, double* eigenvalue,
                                         int32_t* iterations, double* residual)
{
    if (!ctx || !g || !ec) return pg_fail(ctx, PG_ERR_INVALID, "pg_eigen_centrality: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    if (n == 0) {
        if (eigenvalue) *eigenvalue = 0.0;
        if (iterations) *iterations = 0;
        if (residual) *residual = 0.0;
        return PG_OK;
    }
    const bool weighted = g->V != nullptr;
    auto kern = weighted ? k_ec<true> : k_ec<false>;
    const size_t cap = (size_t)ctx->smem_optin - 4096;
    PG_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, EC_THREADS, cap));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "eigenvector kernel cannot be resident");
    const int grid = ctx->sm_count;
    // column blocks as large as the shared memory of the CTA with the most rows allows
    std::vector<int32_t> hR((size_t)n + 1);
    PG_TRY(pg_d2h(ctx, hR.data(), g->R, sizeof(int32_t) * (n + 1)));
    int most = 0;
    for (int r = 0; r < grid; r++)
        most = std::max(most, ec_split(hR.data(), n, r + 1, grid) - ec_split(hR.data(), n, r, grid));
    int cb_log = 0;
    for (int lg = 14; lg >= 8 && !cb_log; lg--)
        if (ec_smem(most, (n + (1 << lg) - 1) >> lg, 1 << lg) <= cap) cb_log = lg;
    if (!cb_log) return pg_fail(ctx, PG_ERR_INTERNAL, "pg_eigen_centrality: %d rows in one block do not fit", most);
    const size_t smem = ec_smem(most, (n + (1 << cb_log) - 1) >> cb_log, 1 << cb_log);
    EcArgs a = {};
    a.R = g->R;
    a.C = g->C;
    a.V = g->V;
    a.n = n;
    a.cb_log = cb_log;
    PG_TRY(pg_wst(ctx, "ec.u0", (size_t)n + 1, &a.u0));
    PG_TRY(pg_wst(ctx, "ec.u1", (size_t)n + 1, &a.u1));
    PG_TRY(pg_wst(ctx, "ec.x", (size_t)n + 1, &a.x_out));
    PG_TRY(pg_wst(ctx, "ec.y", (size_t)n + 1, &a.y_out));
    PG_TRY(pg_wst(ctx, "ec.part", (size_t)grid * 8 + 8, &a.part));
    PG_TRY(pg_wst(ctx, "ec.c16", (size_t)g->nnz + 8, &a.c16));
    PG_TRY(pg_wst(ctx, "ec.info", 4, &a.info));
    double err_sq = EC_EPSILON * EC_EPSILON;   // sqrt(e) > 1e-6 exactly when e > err_sq
    while (std::sqrt(err_sq) > EC_EPSILON) err_sq = std::nextafter(err_sq, 0.0);
    while (std::sqrt(std::nextafter(err_sq, 1.0)) <= EC_EPSILON) err_sq = std::nextafter(err_sq, 1.0);
    a.err_sq = err_sq;
    void* args[] = {(void*)&a};
    PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)kern, dim3(grid), dim3(EC_THREADS), args, smem, ctx->stream));
    PG_LAUNCHED(ctx);
    PG_TRY(pg_d2h(ctx, ec, raw ? a.y_out : a.x_out, sizeof(double) * n));
    double info[3];
    PG_TRY(pg_d2h(ctx, info, a.info, sizeof info));
    if (eigenvalue) *eigenvalue = info[0];
    if (iterations) *iterations = (int32_t)info[1];
    if (residual) *residual = info[2];
    return PG_OK;
}
