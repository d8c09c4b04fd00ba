// bc_dense.cu -- forward Brandes levels as exact integer GEMMs on the
// 5th-generation tensor cores (tcgen05 kind::i8, int32 accumulation in TMEM).
//
// At level d of a 128-source batch, every node v not yet reached by source s
// takes sigma_d[v][s] = sum over neighbours u on level d-1 of s of
// sigma_{d-1}[u][s] (U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:30-50 counts the same
// paths one edge at a time).  With the 0/1 adjacency A (np x np, uint8) and
// X[u][s] = sigma_{d-1}[u][s] on level d-1 (0 elsewhere), that is the
// product A * X.  X is split into 8-bit limbs X = sum_l 256^l X_l; each limb
// product accumulates exactly in int32 (at most np * 255 < 2^31), and the
// epilogue recombines the limbs in 64-bit integers, so sigma is exact and
// equal to the gather kernel's.  On the 58k subject graphs (1 % density,
// ~580 neighbours per node) levels 2 and 3 reach most (node, source) pairs;
// there one pass over the 3.4 GB dense adjacency (HBM-bound, ~0.6 ms) costs
// far less than gathering 1 KB sigma rows for every active neighbour.
//
// Kernel structure: one persistent CTA of 6 warps per SM over 128-row
// tiles.  Warp 0 streams K in 128-byte chunks with TMA (128B swizzle) into a
// ring of 6 (one limb) or 4 (two limbs) stages -- an A tile and one X^T tile
// per limb -- guarded by mbarriers; warp 1 issues 4 UMMA (M=128, N=128,
// K=32) per limb and chunk into one of two TMEM accumulator buffers; warps
// 2-5 read their 32 TMEM lanes (rows) of the finished buffer and update the
// batch state while the next tile's MMAs run.  Every mbarrier wait is
// bounded by the global timer; on expiry the kernel records an error, drains
// its own copies and MMAs, frees TMEM and returns.
#include "bc_dense.cuh"
#include "tma.cuh"
#include <algorithm>

namespace {
using namespace pg_tma;
typedef unsigned long long u64;

constexpr int DM = 128;                     // rows (nodes v) per tile
constexpr int DKC = 128;                    // K bytes (neighbours u) per chunk
constexpr int DS = 128;                     // sources per batch
constexpr uint32_t DTILE = DM * DKC;        // 16 KB per operand tile
// kind::i8 instruction descriptor: S32 accumulator (2 << 4), A and B
// unsigned 8-bit (0), both K-major, N = 128 (>> 3 at bit 17), M = 128 (>> 4 at bit 24)
constexpr uint32_t IDESC_I8 = (2u << 4) | ((uint32_t)(DS >> 3) << 17) | ((uint32_t)(DM >> 4) << 24);

template <int LIMBS>   // 1 or 2 limbs: path counts below 2^16 (max degree < 65536)
struct DCfg {
    static constexpr int STAGES = LIMBS == 1 ? 6 : 4;   // 192 KB of stages either way
    static constexpr uint32_t STAGE = DTILE * (1 + LIMBS);
    static constexpr uint32_t ACC_COLS = LIMBS * DS;                 // one accumulator buffer
    static constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;              // two buffers: 256 or 512
};

struct DCtl {
    u64 full[6];        // stage loaded (TMA complete_tx)
    u64 empty[6];       // stage consumed (MMA commit)
    u64 tfull[2];       // accumulator buffer ready (MMA commit)
    u64 tempty[2];      // accumulator buffer read (one arrive per epilogue warp)
    u64 drainbar;
    long long issued, consumed;
    uint32_t tmem_base;
    int abort;
    int found;
};

template <int LIMBS>
constexpr size_t dsmem() { return 1024 + DCfg<LIMBS>::STAGES * DCfg<LIMBS>::STAGE + sizeof(DCtl) + 64; }

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, u64 a, u64 b, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC_I8), "r"(acc));
}



struct DArgs {
    int n, d;
    u64* sigma;
    int32_t* dist;
    ulonglong2* seen;
    ulonglong2* nxt;
    ulonglong2* fhist;
    double* inv;
    int* flag;
};

// Work units of one launch: tiles [0, nreg) whole (the full rounds of the
// persistent grid); each remaining tail tile split into `spl` parts along K,
// whose int32 partial sums are added (exactly, in any order) into `tail`,
// [tail tile][row][limb column]; k_bc_dense_tail then updates those rows.
struct DUnits {
    int ntiles, nk, nreg, spl;
    int32_t* tail;
    __device__ __forceinline__ int count() const { return nreg + (ntiles - nreg) * spl; }
    // tile of unit u, its chunk range, and its tail index (-1: a whole tile)
    __device__ __forceinline__ void get(int u, int& tile, int& c0, int& c1, int& ti) const
    {
        if (u < nreg) {
            tile = u;
            c0 = 0;
            c1 = nk;
            ti = -1;
            return;
        }
        const int j = u - nreg, part = j % spl;
        ti = j / spl;
        tile = nreg + ti;
        c0 = (int)((long long)nk * part / spl);
        c1 = (int)((long long)nk * (part + 1) / spl);
    }
};

// Level-d update of row v from its path counts: load(cb, r) fills the limb
// values of sources 32 cb .. 32 cb + 31.  Returns true if a source reached v.
template <int LIMBS, class Load>
__device__ __forceinline__ bool update_row(const DArgs& a, int v, Load load)
{
    const bool valid = v < a.n;
    const ulonglong2 sv = valid ? a.seen[v] : make_ulonglong2(0ULL, 0ULL);
    u64 nb0 = 0ULL, nb1 = 0ULL;
#pragma unroll 1
    for (int cb = 0; cb < DS / 32; cb++) {
        uint32_t r[LIMBS][32];
        load(cb, r);
        const u64 seenw = cb < 2 ? sv.x : sv.y;
        const int sh = (cb & 1) * 32;
        uint32_t bits = 0u;
#pragma unroll
        for (int c = 0; c < 32; c++) {
            u64 sg = r[0][c];
            if (LIMBS > 1) sg += (u64)r[1][c] << 8;
            const bool nw = sg != 0ULL && !((seenw >> (sh + c)) & 1ULL);
            if (nw && valid) {
                const size_t at = (size_t)v * DS + cb * 32 + c;
                a.sigma[at] = sg;
                a.dist[at] = a.d;
            }
            bits |= (uint32_t)nw << c;
        }
        if (cb < 2) nb0 |= (u64)bits << sh;
        else nb1 |= (u64)bits << sh;
    }
    if (!valid) return false;
    const ulonglong2 nb = make_ulonglong2(nb0, nb1);
    a.nxt[v] = nb;
    a.seen[v] = make_ulonglong2(sv.x | nb.x, sv.y | nb.y);
    if (a.fhist) a.fhist[v] = nb;
    if (!(nb.x | nb.y)) return false;
    if (a.inv) a.inv[v] += (double)(__popcll(nb.x) + __popcll(nb.y)) / (double)a.d;
    return true;
}

// Warp roles: warp 0 lane 0 streams the operand tiles with TMA, warp 1 lane
// 0 issues the MMAs, warps 2-5 run the epilogue (warp w reads TMEM lanes
// 32 (w % 4) .. + 31).  The accumulator is double-buffered in TMEM, so the
// MMAs of the next unit overlap the epilogue of this one.
constexpr int DWARPS = 6;

template <int LIMBS>
__global__ void __launch_bounds__(DWARPS * 32, 1)
k_bc_dense(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, DUnits un,
           DArgs a, int* __restrict__ err)
{
    using Cfg = DCfg<LIMBS>;
    constexpr int ST = Cfg::STAGES;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    DCtl* ctl = (DCtl*)(smem + ST * Cfg::STAGE);
    volatile int* abort_flag = &ctl->abort;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int units = un.count();
    if (t == 0) {
        for (int s = 0; s < ST; s++) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&ctl->tfull[b], 1);
            mbar_init(&ctl->tempty[b], 4);
        }
        mbar_init(&ctl->drainbar, 1);
        ctl->issued = 0;
        ctl->consumed = 0;
        ctl->abort = 0;
        ctl->found = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&ctl->tmem_base)),
                     "r"(Cfg::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl->tmem_base;

    if (warp == 0) {
        // ---- producer
        if (lane == 0) {
            long long q = 0;
            for (int u = blockIdx.x; u < units && !*abort_flag; u += gridDim.x) {
                int tile, c0, c1, ti;
                un.get(u, tile, c0, c1, ti);
                for (int c = c0; c < c1; c++) {
                    const int s = (int)(q % ST);
                    if (!mbar_wait(&ctl->empty[s], (uint32_t)((q / ST) & 1) ^ 1u) || *abort_flag) {
                        *abort_flag = 1;
                        break;
                    }
                    unsigned char* st = smem + (size_t)s * Cfg::STAGE;
                    mbar_expect_tx(&ctl->full[s], Cfg::STAGE);
                    tma_load(st, &map_a, c * DKC, tile * DM, &ctl->full[s]);
#pragma unroll
                    for (int l = 0; l < LIMBS; l++)
                        tma_load(st + DTILE * (1 + l), &map_b, c * DKC, l * DS, &ctl->full[s]);
                    q++;
                    ctl->issued = q;
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            long long q = 0;
            int tl = 0;
            for (int u = blockIdx.x; u < units && !*abort_flag; u += gridDim.x, tl++) {
                int tile, c0, c1, ti;
                un.get(u, tile, c0, c1, ti);
                const int buf = tl & 1;
                if (!mbar_wait(&ctl->tempty[buf], (uint32_t)((tl >> 1) & 1) ^ 1u)) { *abort_flag = 1; break; }
                tc_fence_after();
                const uint32_t dst = tmem + (uint32_t)(buf * Cfg::ACC_COLS);
                bool ok = true;
                for (int c = c0; c < c1; c++) {
                    const int s = (int)(q % ST);
                    if (!mbar_wait(&ctl->full[s], (uint32_t)((q / ST) & 1)) || *abort_flag) { ok = false; break; }
                    tc_fence_after();
                    unsigned char* st = smem + (size_t)s * Cfg::STAGE;
                    const u64 ad = sdesc(st);
#pragma unroll
                    for (int kk = 0; kk < DKC / 32; kk++) {
                        const u64 o = (u64)(kk * 32) >> 4;   // 32 B per K=32 step
#pragma unroll
                        for (int l = 0; l < LIMBS; l++)
                            umma_i8(dst + (uint32_t)(l * DS), ad + o, sdesc(st + DTILE * (1 + l)) + o,
                                    (c != c0) | (kk != 0));
                    }
                    umma_commit(&ctl->empty[s]);
                    q++;
                    ctl->consumed = q;
                }
                if (!ok) { *abort_flag = 1; break; }
                umma_commit(&ctl->tfull[buf]);
            }
        }
    } else {
        // ---- epilogue: row 32 (warp % 4) + lane of the unit's tile
        const int quarter = warp & 3;
        bool found = false;
        int tl = 0;
        for (int u = blockIdx.x; u < units; u += gridDim.x, tl++) {
            int tile, c0, c1, ti;
            un.get(u, tile, c0, c1, ti);
            const int buf = tl & 1;
            const bool ok = mbar_wait(&ctl->tfull[buf], (uint32_t)((tl >> 1) & 1)) && !*abort_flag;
            if (!ok) {
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const int row = quarter * 32 + lane;
            const uint32_t src = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * Cfg::ACC_COLS);
            if (ti < 0) {
                found |= update_row<LIMBS>(a, tile * DM + row, [&](int cb, uint32_t (&r)[LIMBS][32]) {
#pragma unroll
                    for (int l = 0; l < LIMBS; l++) tmem_ld32(src + (uint32_t)(l * DS + cb * 32), r[l]);
                });
            } else {
                // a part of a tail tile: add its partial sums (exact int32)
                int32_t* dst = un.tail + ((size_t)ti * DM + row) * (LIMBS * DS);
#pragma unroll 1
                for (int l = 0; l < LIMBS; l++)
#pragma unroll 1
                    for (int cb = 0; cb < DS / 32; cb++) {
                        uint32_t r[32];
                        tmem_ld32(src + (uint32_t)(l * DS + cb * 32), r);
#pragma unroll
                        for (int c = 0; c < 32; c++)
                            if (r[c]) atomicAdd(dst + l * DS + cb * 32 + c, (int32_t)r[c]);
                    }
            }
            // the accumulator buffer may be overwritten once every epilogue warp has read it
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->tempty[buf]);
        }
        if (found) ctl->found = 1;
    }
    __syncthreads();
    if (*abort_flag && t == 0) {
        atomicExch(err, 1);
        // wait (bounded) for our own MMAs, then for our own copies still in flight
        umma_commit(&ctl->drainbar);
        mbar_wait(&ctl->drainbar, 0);
        for (long long q = ctl->consumed; q < ctl->issued; q++)
            if (!mbar_wait(&ctl->full[(int)(q % ST)], (uint32_t)((q / ST) & 1))) break;
    }
    tc_fence_before();
    __syncthreads();
    if (t == 0 && ctl->found && a.flag) atomicExch(a.flag, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS));
}

// The rows of the split tail tiles, from their summed partial counts.
template <int LIMBS>
__global__ void k_bc_dense_tail(DUnits un, DArgs a)
{
    const int ntail = un.ntiles - un.nreg;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ntail * DM; g += gridDim.x * blockDim.x) {
        const int ti = g / DM, row = g % DM;
        const int32_t* srcp = un.tail + ((size_t)ti * DM + row) * (LIMBS * DS);
        const bool f = update_row<LIMBS>(a, (un.nreg + ti) * DM + row, [&](int cb, uint32_t (&r)[LIMBS][32]) {
#pragma unroll
            for (int l = 0; l < LIMBS; l++)
#pragma unroll
                for (int c = 0; c < 32; c++) r[l][c] = (uint32_t)srcp[l * DS + cb * 32 + c];
        });
        if (f && a.flag) atomicExch(a.flag, 1);
    }
}

// X^T for level d: row l * 128 + s holds limb l of sigma[u][s] for u on
// level d - 1 of source s (0 elsewhere).  A block transposes 64 nodes x 128
// sources through shared memory: coalesced sigma rows in, 64-byte row runs out.
template <int LIMBS>
__global__ void __launch_bounds__(256)
k_bc_xt(const u64* __restrict__ sigma, const ulonglong2* __restrict__ fprev, int n, int np, uint8_t* __restrict__ xt)
{
    __shared__ uint32_t tile[LIMBS][DS][64 / 4 + 1];
    const int u0 = blockIdx.x * 64;
    for (int e = threadIdx.x; e < LIMBS * DS * 16; e += blockDim.x) (&tile[0][0][0])[(e / 16) * 17 + (e % 16)] = 0u;
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * DS; e += blockDim.x) {
        const int ul = e >> 7, s = e & (DS - 1), u = u0 + ul;
        u64 sg = 0ULL;
        if (u < n) {
            const ulonglong2 m = fprev[u];
            const u64 w = s < 64 ? m.x : m.y;
            if ((w >> (s & 63)) & 1ULL) sg = sigma[(size_t)u * DS + s];
        }
        if (sg) {
#pragma unroll
            for (int l = 0; l < LIMBS; l++) {
                const uint32_t b = (uint32_t)((sg >> (8 * l)) & 255ULL);
                if (b) atomicOr(&tile[l][s][ul >> 2], b << (8 * (ul & 3)));
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < LIMBS * DS * 16; e += blockDim.x) {
        const int row = e >> 4, w = e & 15;
        const int l = row / DS, s = row % DS;
        *(uint32_t*)(xt + (size_t)(l * DS + s) * np + u0 + 4 * w) = tile[l][s][w];
    }
}

__global__ void k_bc_adj(const int32_t* __restrict__ R, const int32_t* __restrict__ C, int n, int np,
                         uint8_t* __restrict__ adj)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int v = warp; v < n; v += nw)
        for (int q = R[v] + lane; q < R[v + 1]; q += 32) adj[(size_t)v * np + C[q]] = 1;
}

bool make_map_u8(CUtensorMap* m, const uint8_t* base, int rows, int cols)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols};
    cuuint32_t box[2] = {(cuuint32_t)DKC, (cuuint32_t)DM};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

template <int LIMBS>
pg_status launch_level(pg_ctx* ctx, BCDense& d, const BCLevel& lv, int* err)
{
    const int nb = d.np / DM, nk = d.np / DKC;
    k_bc_xt<LIMBS><<<d.np / 64, 256, 0, ctx->stream>>>(lv.sigma, lv.fprev, d.n, d.np, d.xt);
    PG_LAUNCHED(ctx);
    CUtensorMap map_b;
    if (!make_map_u8(&map_b, d.xt, LIMBS * DS, d.np))
        return pg_fail(ctx, PG_ERR_CUDA, "cuTensorMapEncodeTiled failed for the Brandes level operand");
    DArgs a;
    a.n = d.n;
    a.d = lv.d;
    a.sigma = lv.sigma;
    a.dist = lv.dist;
    a.seen = lv.seen;
    a.nxt = lv.nxt;
    a.fhist = lv.fhist;
    a.inv = lv.inv;
    a.flag = lv.flag;
    const int grid = std::min(ctx->sm_count, nb);
    // whole tiles for the full rounds of the grid; the last partial round's
    // tiles split along K over the idle CTAs (at least 8 chunks per part)
    DUnits un;
    un.ntiles = nb;
    un.nk = nk;
    un.nreg = nb / grid * grid;
    un.spl = 1;
    un.tail = d.tail;
    const int ntail = nb - un.nreg;
    if (un.nreg > 0 && ntail > 0) un.spl = std::max(1, std::min(grid / ntail, nk / 8));
    if (un.spl == 1) un.nreg = nb;   // no split: every tile whole
    else PG_CUDA(ctx, cudaMemsetAsync(d.tail, 0, sizeof(int32_t) * (size_t)ntail * DM * LIMBS * DS, ctx->stream));
    const size_t smem = dsmem<LIMBS>();
    PG_CUDA(ctx, cudaFuncSetAttribute(k_bc_dense<LIMBS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int prof = pg_prof_begin(ctx, "k_bc_dense");
    k_bc_dense<LIMBS><<<grid, DWARPS * 32, smem, ctx->stream>>>(d.map_adj, map_b, un, a, err);
    PG_LAUNCHED(ctx);
    if (un.nreg < nb) {
        k_bc_dense_tail<LIMBS><<<ceil_div((long long)ntail * DM, 128), 128, 0, ctx->stream>>>(un, a);
        PG_LAUNCHED(ctx);
    }
    pg_prof_end(ctx, prof);
    return PG_OK;
}
}  // namespace

bool bc_dense_eligible(pg_ctx* ctx, int n, long long nnz, int max_deg)
{
    if (n < 2 * DM || !encode_fn()) return false;
    if (max_deg >= 65536) return false;             // level-2 path counts fit two 8-bit limbs
    if ((size_t)ctx->smem_optin < dsmem<2>()) return false;
    const long long np = (n + DM - 1) / DM * DM;
    if (np * np > (8LL << 30)) return false;        // adjacency of at most 8 GiB
    if (nnz < 64LL * n) return false;               // rows of at least 64 neighbours on average
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (size_t)(np * np) * 2 < free_b;
}

pg_status bc_dense_setup(pg_ctx* ctx, const int32_t* R, const int32_t* C, int n, BCDense& d)
{
    d.n = n;
    d.np = (n + DM - 1) / DM * DM;
    const size_t np = (size_t)d.np;
    PG_TRY(pg_wst(ctx, "bc.adj", np * np, &d.adj));
    PG_TRY(pg_wst(ctx, "bc.xt", 2 * DS * np, &d.xt));
    PG_TRY(pg_wst(ctx, "bc.dense_err", 1, &d.err));
    // partial sums of tail tiles: fewer tail tiles than SMs, two limbs at most
    PG_TRY(pg_wst(ctx, "bc.dense_tail", (size_t)std::max(ctx->sm_count, 1) * DM * 2 * DS, &d.tail));
    PG_CUDA(ctx, cudaMemsetAsync(d.err, 0, sizeof(int), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(d.adj, 0, np * np, ctx->stream));
    k_bc_adj<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(R, C, n, d.np, d.adj);
    PG_LAUNCHED(ctx);
    if (!make_map_u8(&d.map_adj, d.adj, d.np, d.np))
        return pg_fail(ctx, PG_ERR_CUDA, "cuTensorMapEncodeTiled failed for the dense adjacency");
    return PG_OK;
}

pg_status bc_dense_check(pg_ctx* ctx, BCDense& d)
{
    int herr = 0;
    PG_TRY(pg_d2h(ctx, &herr, d.err, sizeof(int)));
    if (herr) return pg_fail(ctx, PG_ERR_TIMEOUT, "dense Brandes level: a pipeline wait timed out");
    return PG_OK;
}

pg_status bc_dense_level(pg_ctx* ctx, BCDense& d, const BCLevel& lv)
{
    int* err = d.err;
    // sigma on level d - 1 is at most max_deg^(d - 2) (1 on level 1)
    double bound = 1.0;
    for (int k = 2; k < lv.d; k++) bound *= (double)std::max(d.max_deg, 1);
    if (bound < 256.0) return launch_level<1>(ctx, d, lv, err);
    if (bound < 65536.0) return launch_level<2>(ctx, d, lv, err);
    return pg_fail(ctx, PG_ERR_INTERNAL, "dense Brandes level %d: path counts need more than 16 bits", lv.d);
}
