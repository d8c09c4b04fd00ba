// maslov.cu -- Maslov-Sneppen degree-preserving rewiring (Rewire / Maslov,
// U/cuda_EC/cuda_EC/Maslov.cpp:8-109; Maslov_weighted_1,
// W/Maslov/Maslov/Maslov.cpp:50-196).
//
// The reference runs 2M sequential attempts drawn from rand().  Here the
// attempts come from a seeded counter-based generator and run in rounds of
// B attempts: every attempt of a round reads the state left by the previous
// round (two random edge slots, the swap orientation coin, the shared
// end-point test and the "new edge already exists" test against an N x N
// edge bitmap), valid attempts claim their four end points with atomicMin of
// the attempt index, and only attempts that own all four commit.  Committed
// attempts of one round touch disjoint vertices (hence disjoint slots and
// bitmap bits), so the round's result does not depend on thread timing and
// equals the sequential restatement in the oracle bit for bit.
// Weights stay with the edge slot that carries them, as in Maslov_weighted_1.
#include "pg_internal.cuh"
#include <algorithm>

namespace {
__device__ __host__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ bool has_edge(const unsigned long long* bits, uint64_t n, int a, int b)
{
    uint64_t q = (uint64_t)a * n + (uint64_t)b;
    return (bits[q >> 6] >> (q & 63)) & 1ULL;
}
__device__ __forceinline__ void put_edge(unsigned long long* bits, uint64_t n, int a, int b, bool on)
{
    uint64_t q = (uint64_t)a * n + (uint64_t)b;
    unsigned long long m = 1ULL << (q & 63);
    if (on) atomicOr(&bits[q >> 6], m); else atomicAnd(&bits[q >> 6], ~m);
}

// Upper-triangle edge slots from the CSR (row-major order, as the
// reference's E array) and the edge bitmap.
__global__ void k_ms_init(const int32_t* __restrict__ R, const int32_t* __restrict__ C, const float* __restrict__ V,
                          int32_t n, const long long* __restrict__ upper_off, int* __restrict__ ea,
                          int* __restrict__ eb, float* __restrict__ ew, unsigned long long* __restrict__ bits)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        long long pos = upper_off[i];
        for (int32_t base = R[i]; base < R[i + 1]; base += 32) {
            int32_t q = base + lane;
            bool up = false;
            int c = 0;
            if (q < R[i + 1]) {
                c = C[q];
                put_edge(bits, (uint64_t)n, i, c, true);
                up = c > i;
            }
            unsigned m = __ballot_sync(0xffffffffu, up);
            if (up) {
                long long s = pos + __popc(m & ((1u << lane) - 1u));
                ea[s] = i;
                eb[s] = c;
                ew[s] = V ? V[q] : 1.0f;
            }
            pos += __popc(m);
        }
    }
}

__global__ void k_ms_upper_count(const int32_t* __restrict__ R, const int32_t* __restrict__ C, int32_t n,
                                 int32_t* __restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        int c = 0;
        for (int32_t q = R[i] + lane; q < R[i + 1]; q += 32) c += C[q] > i;
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) cnt[i] = c;
    }
}

struct Attempt {
    int v[4];
    long long i, j;
    int ok, coin;
};

__global__ void k_ms_propose(const int* __restrict__ ea, const int* __restrict__ eb, long long M, int32_t n,
                             const unsigned long long* __restrict__ bits, uint64_t seed, long long base, int nb,
                             Attempt* __restrict__ at, unsigned int* __restrict__ owner)
{
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) {
        uint64_t idx = (uint64_t)(base + a);
        uint64_t h1 = mix64(seed ^ (2 * idx)), h2 = mix64(seed ^ (2 * idx + 1));
        long long i = (long long)(h1 % (uint64_t)M), j = (long long)(h2 % (uint64_t)M);
        int c = (int)((h1 >> 63) ^ (h2 >> 63));
        int V1 = ea[i], V2 = eb[i], V3 = ea[j], V4 = eb[j];
        bool ok = !(V1 == V3 || V1 == V4 || V2 == V3 || V2 == V4);
        if (ok) {
            if (c) ok = !(has_edge(bits, n, V1, V3) || has_edge(bits, n, V2, V4));
            else ok = !(has_edge(bits, n, V1, V4) || has_edge(bits, n, V2, V3));
        }
        Attempt t;
        t.v[0] = V1; t.v[1] = V2; t.v[2] = V3; t.v[3] = V4;
        t.i = i; t.j = j; t.ok = ok; t.coin = c;
        at[a] = t;
        if (ok)
            for (int q = 0; q < 4; q++) atomicMin(&owner[t.v[q]], (unsigned)a);
    }
}

__global__ void k_ms_commit(const Attempt* __restrict__ at, int nb, int32_t n, const unsigned int* __restrict__ owner,
                            int* __restrict__ ea, int* __restrict__ eb, unsigned long long* __restrict__ bits,
                            unsigned long long* __restrict__ committed)
{
    unsigned long long mine = 0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) {
        Attempt t = at[a];
        if (!t.ok) continue;
        bool own = true;
        for (int q = 0; q < 4; q++) own &= owner[t.v[q]] == (unsigned)a;
        if (!own) continue;
        int V1 = t.v[0], V2 = t.v[1], V3 = t.v[2], V4 = t.v[3];
        put_edge(bits, n, V1, V2, false); put_edge(bits, n, V2, V1, false);
        put_edge(bits, n, V3, V4, false); put_edge(bits, n, V4, V3, false);
        if (t.coin) {  // 1-3, 2-4 (Maslov.cpp:31-42)
            put_edge(bits, n, V1, V3, true); put_edge(bits, n, V3, V1, true);
            put_edge(bits, n, V2, V4, true); put_edge(bits, n, V4, V2, true);
            eb[t.i] = V3;
            ea[t.j] = V2;
        } else {       // 1-4, 3-2 (Maslov.cpp:44-55)
            put_edge(bits, n, V1, V4, true); put_edge(bits, n, V4, V1, true);
            put_edge(bits, n, V2, V3, true); put_edge(bits, n, V3, V2, true);
            eb[t.i] = V4;
            eb[t.j] = V2;
        }
        mine++;
    }
    mine = __reduce_add_sync(0xffffffffu, (unsigned)mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(committed, mine);
}

__global__ void k_ms_release(const Attempt* __restrict__ at, int nb, unsigned int* __restrict__ owner)
{
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) {
        Attempt t = at[a];
        if (t.ok)
            for (int q = 0; q < 4; q++) owner[t.v[q]] = 0xffffffffu;
    }
}

__global__ void k_ms_pairs(const int* __restrict__ ea, const int* __restrict__ eb, long long M, int2* __restrict__ p)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M; q += (long long)gridDim.x * blockDim.x)
        p[q] = make_int2(ea[q], eb[q]);
}
}  // namespace

extern "C" int64_t pg_maslov_round_size(int64_t M)
{
    int64_t b = M / 16;
    if (b < 1) b = 1;
    if (b > 65536) b = 65536;
    return b;
}

extern "C" pg_status pg_maslov(pg_ctx* ctx, const pg_graph* g, uint64_t seed, int64_t attempts, pg_graph** out,
                               int64_t* committed)
{
    if (!ctx || !g || !out || attempts < 0) return pg_fail(ctx, PG_ERR_INVALID, "pg_maslov: bad arguments");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    const long long M = g->nnz / 2;
    int32_t* cnt;
    long long* off;
    int *ea, *eb;
    float* ew;
    unsigned long long *bits, *ncommit;
    unsigned int* owner;
    Attempt* at;
    const uint64_t nbits = (uint64_t)n * (uint64_t)n;
    const size_t words = (size_t)((nbits + 63) / 64);
    const long long B = pg_maslov_round_size(M);
    PG_TRY(pg_wst(ctx, "ms.cnt", (size_t)n + 1, &cnt));
    PG_TRY(pg_wst(ctx, "ms.off", (size_t)n + 2, &off));
    PG_TRY(pg_wst(ctx, "ms.ea", (size_t)M + 1, &ea));
    PG_TRY(pg_wst(ctx, "ms.eb", (size_t)M + 1, &eb));
    PG_TRY(pg_wst(ctx, "ms.ew", (size_t)M + 1, &ew));
    PG_TRY(pg_wst(ctx, "ms.bits", words + 1, &bits));
    PG_TRY(pg_wst(ctx, "ms.owner", (size_t)n + 1, &owner));
    PG_TRY(pg_wst(ctx, "ms.at", (size_t)B, &at));
    PG_TRY(pg_wst(ctx, "ms.ncommit", 1, &ncommit));
    PG_CUDA(ctx, cudaMemsetAsync(bits, 0, sizeof(unsigned long long) * words, ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(owner, 0xff, sizeof(unsigned int) * (n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(ncommit, 0, sizeof(unsigned long long), ctx->stream));
    const int grid = ctx->sm_count * 4;
    k_ms_upper_count<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, n, cnt);
    PG_LAUNCHED(ctx);
    PG_TRY(pg_scan_counts(ctx, cnt, (int64_t*)off, n));
    k_ms_init<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, g->V, n, off, ea, eb, ew, bits);
    PG_LAUNCHED(ctx);
    if (M >= 2) {
        for (long long base = 0; base < attempts; base += B) {
            int nb = (int)std::min<long long>(B, attempts - base);
            int gr = std::max(1, std::min(grid, ceil_div(nb, 256)));
            k_ms_propose<<<gr, 256, 0, ctx->stream>>>(ea, eb, M, n, bits, seed, base, nb, at, owner);
            PG_LAUNCHED(ctx);
            k_ms_commit<<<gr, 256, 0, ctx->stream>>>(at, nb, n, owner, ea, eb, bits, ncommit);
            PG_LAUNCHED(ctx);
            k_ms_release<<<gr, 256, 0, ctx->stream>>>(at, nb, owner);
            PG_LAUNCHED(ctx);
        }
    }
    int2* pairs;
    PG_TRY(pg_wst(ctx, "ms.pairs", (size_t)M + 1, &pairs));
    k_ms_pairs<<<grid, 256, 0, ctx->stream>>>(ea, eb, M, pairs);
    PG_LAUNCHED(ctx);
    PG_TRY(pg_csr_from_pairs(ctx, n, pairs, g->V ? ew : nullptr, M, out));
    if (committed) {
        unsigned long long c;
        PG_TRY(pg_d2h(ctx, &c, ncommit, sizeof c));
        *committed = (int64_t)c;
    }
    return PG_OK;
}
