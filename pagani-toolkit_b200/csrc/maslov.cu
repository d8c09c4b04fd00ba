// maslov.cu -- Maslov-Sneppen degree-preserving rewiring (Rewire / Maslov,
// U/cuda_EC/cuda_EC/Maslov.cpp:8-109; Maslov_weighted_1,
// W/Maslov/Maslov/Maslov.cpp:50-196).
//
// The reference evaluates its swap attempts one after another, each on the
// graph the previous ones left: two random edge slots i, j (edges 1-2 and
// 3-4), a coin for the new pairing (1-3 + 2-4, or 1-4 + 3-2), rejection when
// the edges share an end point or a new edge already exists, otherwise the
// swap is applied to the slots and to the adjacency matrix.
//
// Here the attempts come from a seeded counter-based generator (attempt a
// uses bits 2a and 2a + 1 of a splitmix64 stream keyed by the seed) and are
// evaluated in rounds, all attempts of a round on the state the previous
// round left:
//   - a valid attempt claims its two slots and its two new pairs, lowest
//     attempt index first (atomicMin of the index relative to the round's
//     oldest attempt; slots in an owner array, pairs in a direct-mapped table
//     where a collision of two pairs only costs a deferral); attempts that
//     own all four claims commit;
//   - every valid attempt that lost a claim is deferred to the next round
//     and evaluated again there, and so is every rejected attempt whose
//     evaluation read something a lower-index attempt of the round may
//     write: a slot or a checked pair entry that a lower-index valid attempt
//     claimed (conservative: that attempt may not commit), or a checked pair
//     that a lower-index commit removes (committers record the pairs they
//     remove); the other rejected attempts are decided.
// Each decided attempt thus saw exactly the state the lower-index commits of
// its round leave (commits touch disjoint slots and create distinct pairs,
// and a valid attempt's new pairs are absent from the round's state), so a
// round is the reference's sequential chain over its decided attempts in
// index order, and every requested attempt is decided once.  Measured
// against the reference's own Maslov (compiled from its sources, 100 seeds),
// the committed fraction and the surrogates' clustering agree in
// distribution (tests/test_maslov_reference_cpu.py).  The decisions depend
// only on the state and the indices, not on thread timing, and equal the
// oracle's sequential restatement (or_maslov) bit for bit.
//
// All rounds run in one cooperative launch with grid-wide barriers between
// the evaluate / commit / release phases; the round counters live in a
// device control block, so the launch needs no host round trip and can be
// captured in a CUDA graph.  Weights stay with their edge slot, as in
// Maslov_weighted_1.
#include "pg_internal.cuh"
#include "maslov.cuh"
#include <algorithm>
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

namespace cg = cooperative_groups;

namespace {
constexpr int MS_THREADS = 256;

__device__ __host__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Edge bitmap over the unordered pairs {a, b}, a != b: bit lo (2n - lo - 1) / 2
// + (hi - lo - 1), n(n - 1)/2 bits.
__device__ __forceinline__ uint64_t pair_bit(uint64_t n, int a, int b)
{
    const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    return lo * (2 * n - lo - 1) / 2 + (hi - lo - 1);
}
__device__ __forceinline__ bool has_edge(const unsigned long long* bits, uint64_t n, int a, int b)
{
    const uint64_t q = pair_bit(n, a, b);
    return (bits[q >> 6] >> (q & 63)) & 1ULL;
}
__device__ __forceinline__ void put_edge(unsigned long long* bits, uint64_t n, int a, int b, bool on)
{
    const uint64_t q = pair_bit(n, a, b);
    const unsigned long long m = 1ULL << (q & 63);
    if (on) atomicOr(&bits[q >> 6], m); else atomicAnd(&bits[q >> 6], ~m);
}

// table entry of the unordered pair {a, b}
__device__ __host__ __forceinline__ uint32_t pair_slot(int a, int b, uint64_t n, uint32_t hmask)
{
    uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
    return (uint32_t)(mix64(lo * n + hi) & hmask);
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
                up = c > i;
                if (up) put_edge(bits, (uint64_t)n, i, c, true);
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

__global__ void k_ms_reset(MsControl* __restrict__ st, uint64_t attempts, unsigned long long* __restrict__ slot_owner,
                           long long M, unsigned long long* __restrict__ table, unsigned long long* __restrict__ pair_wr,
                           uint32_t hsize)
{
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    for (long long q = tid; q < M; q += nt) slot_owner[q] = ~0ULL;
    for (long long q = tid; q < hsize; q += nt) table[q] = pair_wr[q] = ~0ULL;
    if (tid == 0) {
        st->n_pending[0] = st->n_pending[1] = 0;
        st->oldest[0] = st->oldest[1] = ~0ULL;
        st->committed = 0;
        st->rounds = 0;
    }
}

struct MsItem {
    unsigned long long a;   // attempt index
    int v[4];
    int i, j;               // slots
    uint32_t h[2];          // table entries of the new pairs
    int state;              // 0 shared end point, 1 new edge exists, 2 valid, 3 committing
    int coin;
};

__device__ __forceinline__ uint64_t stream_key(uint64_t seed) { return mix64(seed ^ 0xD1B54A32D192ED03ULL); }
__device__ __forceinline__ uint64_t stream_bits(uint64_t key, uint64_t q)
{
    return mix64(key + q * 0x9E3779B97F4A7C15ULL);
}

// Defers attempt a to the next round.  The threads deferring together
// append with one atomic (their order in the list does not matter: claims
// are ordered by attempt index), and fold the oldest deferred attempt with
// one atomicMin; one atomic per deferred attempt on these two counters
// serialised in L2.
__device__ __forceinline__ void ms_defer(unsigned long long a, unsigned long long base, MsControl* st, int slot,
                                         unsigned long long* pnext)
{
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long at = 0;
    if (g.thread_rank() == 0) at = atomicAdd(&st->n_pending[slot], (unsigned long long)g.size());
    at = g.shfl(at, 0) + g.thread_rank();
    pnext[at] = a;
    const unsigned rel = cg::reduce(g, (unsigned)(a - base), cg::less<unsigned>());
    if (g.thread_rank() == 0) atomicMin(&st->oldest[slot], base + rel);
}

__global__ void __launch_bounds__(MS_THREADS, 4)   // four CTAs per SM: at most two attempts per thread a round
k_ms_rounds(MsArgs p)
{
    cg::grid_group grid = cg::this_grid();
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    const uint64_t n = (uint64_t)p.n;
    const uint64_t key = stream_key(p.seed_dev ? p.seed_dev[*p.round_dev] : p.seed);
    unsigned long long* pend = p.pend_a;
    unsigned long long* pnext = p.pend_b;
    MsItem* items = (MsItem*)p.items;
    volatile MsControl* vst = p.st;
    // Claims and write records are 64-bit (round tag << 32 | attempt index
    // relative to the round's oldest); the tag decreases with the round, so
    // this round's entries are below every older one and nothing needs to be
    // cleared between rounds.
    unsigned long long fresh = 0;
    unsigned long long committed = 0;   // this thread's commits, added once at the end
    for (uint32_t round = 0;; round++) {
        const int cur = round & 1;
        const unsigned long long np = vst->n_pending[cur];
        const unsigned long long take = min(p.attempts - fresh, (unsigned long long)p.B - np);
        const unsigned long long total = np + take;
        if (total == 0) break;                                   // uniform over the grid
        const unsigned long long base = np ? vst->oldest[cur] : fresh;   // oldest attempt of the round
        const unsigned long long tag = (unsigned long long)(0xffffffffu - round) << 32;
        if (tid == 0) {           // the next round's counters (last read one round ago)
            p.st->n_pending[cur ^ 1] = 0;
            p.st->oldest[cur ^ 1] = ~0ULL;
        }
        // Every phase takes a thread's attempts two at a time and issues the
        // loads of both before either result is used: a round has more
        // attempts than resident threads, and the barrier after each phase
        // waits for the threads with two dependent memory chains.  Within a
        // phase no attempt writes what another reads, so the order inside a
        // thread changes nothing.
        // ---- evaluate on the round's state; valid attempts claim
        for (long long it0 = tid; it0 < (long long)total; it0 += 2 * nt) {
            MsItem t[2];
            bool ok[2], shared[2], e1[2], e2[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const long long it = it0 + k * nt;
                ok[k] = it < (long long)total;
                const long long ic = ok[k] ? it : it0;   // an idle half repeats the first attempt's reads
                t[k].a = ic < (long long)np ? pend[ic] : fresh + (ic - np);
                const uint64_t h1 = stream_bits(key, 2 * t[k].a), h2 = stream_bits(key, 2 * t[k].a + 1);
                t[k].i = (int)(h1 % (uint64_t)p.M);
                t[k].j = (int)(h2 % (uint64_t)p.M);
                t[k].coin = (int)((h1 >> 63) ^ (h2 >> 63));
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                t[k].v[0] = p.ea[t[k].i]; t[k].v[1] = p.eb[t[k].i]; t[k].v[2] = p.ea[t[k].j]; t[k].v[3] = p.eb[t[k].j];
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int x1 = t[k].v[0], x2 = t[k].coin ? t[k].v[2] : t[k].v[3];   // new pair 1: 1-3 or 1-4
                const int y1 = t[k].v[1], y2 = t[k].coin ? t[k].v[3] : t[k].v[2];   // new pair 2: 2-4 or 2-3
                t[k].h[0] = pair_slot(x1, x2, n, p.hmask);
                t[k].h[1] = pair_slot(y1, y2, n, p.hmask);
                shared[k] = t[k].v[0] == t[k].v[2] || t[k].v[0] == t[k].v[3] || t[k].v[1] == t[k].v[2] ||
                            t[k].v[1] == t[k].v[3];
                // both probes (only of distinct end points, which the bitmap indexes)
                e1[k] = !shared[k] && has_edge(p.bits, n, x1, x2);
                e2[k] = !shared[k] && has_edge(p.bits, n, y1, y2);
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (!ok[k]) continue;
                t[k].state = shared[k] ? 0 : (e1[k] || e2[k]) ? 1 : 2;
                if (t[k].state == 2) {
                    const unsigned long long me = tag | (uint32_t)(t[k].a - base);
                    atomicMin(&p.slot_owner[t[k].i], me);
                    atomicMin(&p.slot_owner[t[k].j], me);
                    atomicMin(&p.table[t[k].h[0]], me);
                    atomicMin(&p.table[t[k].h[1]], me);
                }
                items[it0 + k * nt] = t[k];
            }
        }
        grid.sync();
        // ---- valid attempts owning all four claims commit (their writes are
        // recorded, then applied); valid attempts that lost are deferred
        unsigned long long mine = 0;
        for (long long it0 = tid; it0 < (long long)total; it0 += 2 * nt) {
            MsItem t[2];
            bool ok[2];
            unsigned long long c[2][4];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const long long it = it0 + k * nt;
                ok[k] = it < (long long)total;
                t[k] = items[ok[k] ? it : it0];
                ok[k] = ok[k] && t[k].state == 2;
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                c[k][0] = p.slot_owner[t[k].i];
                c[k][1] = p.slot_owner[t[k].j];
                c[k][2] = p.table[t[k].h[0]];
                c[k][3] = p.table[t[k].h[1]];
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (!ok[k]) continue;
                const unsigned long long me = tag | (uint32_t)(t[k].a - base);
                if (!(c[k][0] == me && c[k][1] == me && c[k][2] == me && c[k][3] == me)) {
                    ms_defer(t[k].a, base, p.st, cur ^ 1, pnext);
                    continue;
                }
                atomicMin(&p.pair_wr[pair_slot(t[k].v[0], t[k].v[1], n, p.hmask)], me);   // the pairs it removes
                atomicMin(&p.pair_wr[pair_slot(t[k].v[2], t[k].v[3], n, p.hmask)], me);
                const int V1 = t[k].v[0], V2 = t[k].v[1], V3 = t[k].v[2], V4 = t[k].v[3];
                put_edge(p.bits, n, V1, V2, false);
                put_edge(p.bits, n, V3, V4, false);
                if (t[k].coin) {   // 1-3, 2-4 (Maslov.cpp:36-44)
                    put_edge(p.bits, n, V1, V3, true);
                    put_edge(p.bits, n, V2, V4, true);
                    p.eb[t[k].i] = V3;
                    p.ea[t[k].j] = V2;
                } else {        // 1-4, 3-2 (Maslov.cpp:47-56)
                    put_edge(p.bits, n, V1, V4, true);
                    put_edge(p.bits, n, V2, V3, true);
                    p.eb[t[k].i] = V4;
                    p.eb[t[k].j] = V2;
                }
                mine++;
            }
        }
        committed += mine;
        grid.sync();
        // ---- a rejected attempt is deferred when a lower-index valid attempt
        // claimed one of its slots or a pair entry it checked, or a lower-index
        // commit removes a pair it checked (conservative: the claimant may not
        // have committed)
        for (long long it0 = tid; it0 < (long long)total; it0 += 2 * nt) {
            MsItem t[2];
            bool ok[2];
            unsigned long long c[2][6];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const long long it = it0 + k * nt;
                ok[k] = it < (long long)total;
                t[k] = items[ok[k] ? it : it0];
                ok[k] = ok[k] && t[k].state < 2;
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                c[k][0] = p.slot_owner[t[k].i];
                c[k][1] = p.slot_owner[t[k].j];
                const bool chk = t[k].state == 1;
                c[k][2] = chk ? p.table[t[k].h[0]] : ~0ULL;
                c[k][3] = chk ? p.table[t[k].h[1]] : ~0ULL;
                c[k][4] = chk ? p.pair_wr[t[k].h[0]] : ~0ULL;
                c[k][5] = chk ? p.pair_wr[t[k].h[1]] : ~0ULL;
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (!ok[k]) continue;
                const unsigned long long me = tag | (uint32_t)(t[k].a - base);
                const bool defer = c[k][0] < me || c[k][1] < me || c[k][2] < me || c[k][3] < me || c[k][4] < me ||
                                   c[k][5] < me;
                if (defer) ms_defer(t[k].a, base, p.st, cur ^ 1, pnext);
            }
        }
        fresh += take;
        if (tid == 0) p.st->rounds = round + 1;
        grid.sync();
        unsigned long long* tmp = pend;
        pend = pnext;
        pnext = tmp;
    }
    committed = __reduce_add_sync(0xffffffffu, (unsigned)committed);
    if ((threadIdx.x & 31) == 0 && committed) atomicAdd(&p.st->committed, committed);
}

// Rows of the rewired graph: R is unchanged (degrees are preserved), so each
// slot's two directions are scattered behind per-row cursors and the rows are
// then sorted (launch_row_sort), carrying the slot's weight.
__global__ void k_ms_cursor(const int32_t* __restrict__ R, int32_t n, int32_t* __restrict__ cur)
{
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) cur[v] = R[v];
}

__global__ void k_ms_scatter(const int* __restrict__ ea, const int* __restrict__ eb, const float* __restrict__ ew,
                             long long M, int32_t* __restrict__ cur, int32_t* __restrict__ Ct, float* __restrict__ Vt)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M; q += (long long)gridDim.x * blockDim.x) {
        const int a = ea[q], b = eb[q];
        const int32_t pa = atomicAdd(&cur[a], 1), pb = atomicAdd(&cur[b], 1);
        Ct[pa] = b;
        Ct[pb] = a;
        if (Vt) {
            Vt[pa] = ew[q];
            Vt[pb] = ew[q];
        }
    }
}
}  // namespace

int64_t ms_round_size(int64_t M)
{
    int64_t b = M / 32;
    if (b < 64) b = 64;
    if (b > (1LL << 20)) b = 1LL << 20;
    return b;
}

uint32_t ms_table_size(int64_t B)
{
    uint32_t h = 1024;
    while ((int64_t)h < 64 * B) h <<= 1;
    return h;
}

pg_status ms_prepare(pg_ctx* ctx, const pg_graph* g, uint64_t seed, int64_t attempts, MsArgs* a)
{
    const int n = g->n;
    const long long M = g->nnz / 2;
    const long long B = ms_round_size(M);
    const uint32_t H = ms_table_size(B);
    const uint64_t nbits = (uint64_t)n * (uint64_t)(n > 0 ? n - 1 : 0) / 2;   // unordered pairs
    const size_t words = (size_t)((nbits + 63) / 64);
    memset(a, 0, sizeof *a);
    a->n = n;
    a->M = M;
    a->B = B;
    a->hmask = H - 1;
    a->seed = seed;
    PG_TRY(pg_wst(ctx, "ms.cnt", (size_t)n + 1, &a->cnt));
    PG_TRY(pg_wst(ctx, "ms.off", (size_t)n + 2, &a->off));
    PG_TRY(pg_wst(ctx, "ms.ea", (size_t)M + 1, &a->ea));
    PG_TRY(pg_wst(ctx, "ms.eb", (size_t)M + 1, &a->eb));
    PG_TRY(pg_wst(ctx, "ms.ew", (size_t)M + 1, &a->ew));
    PG_TRY(pg_wst(ctx, "ms.bits", words + 1, &a->bits));
    PG_TRY(pg_wst(ctx, "ms.slot_owner", (size_t)M + 1, &a->slot_owner));
    PG_TRY(pg_wst(ctx, "ms.table", (size_t)H, &a->table));
    PG_TRY(pg_wst(ctx, "ms.pair_wr", (size_t)H, &a->pair_wr));
    PG_TRY(pg_wst(ctx, "ms.items", (size_t)B, (MsItem**)&a->items));
    PG_TRY(pg_wst(ctx, "ms.pend_a", (size_t)B, &a->pend_a));
    PG_TRY(pg_wst(ctx, "ms.pend_b", (size_t)B, &a->pend_b));
    PG_TRY(pg_wst(ctx, "ms.ctl", 1, &a->st));
    PG_TRY(pg_wst(ctx, "ms.cursor", (size_t)n + 1, &a->cursor));
    PG_TRY(pg_wst(ctx, "ms.ct", (size_t)(2 * M) + 1, &a->ct));
    if (g->V) PG_TRY(pg_wst(ctx, "ms.vt", (size_t)(2 * M) + 1, &a->vt));
    a->words = words;
    a->attempts = (uint64_t)attempts;
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ms_rounds, MS_THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "maslov: kernel does not fit an SM");
    a->grid = ctx->sm_count * std::min(per_sm, 4);
    return PG_OK;
}

// Enqueues the whole rewiring on the context stream: no host round trip, no
// allocation (ms_prepare sized the workspace).
pg_status ms_enqueue(pg_ctx* ctx, const pg_graph* g, MsArgs* a)
{
    const int grid = ctx->sm_count * 4;
    PG_CUDA(ctx, cudaMemsetAsync(a->bits, 0, sizeof(unsigned long long) * a->words, ctx->stream));
    k_ms_reset<<<grid, 256, 0, ctx->stream>>>(a->st, a->attempts, a->slot_owner, a->M, a->table, a->pair_wr,
                                               a->hmask + 1);
    PG_LAUNCHED(ctx);
    k_ms_upper_count<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, a->n, a->cnt);
    PG_LAUNCHED(ctx);
    PG_TRY(pg_scan_counts(ctx, a->cnt, (int64_t*)a->off, a->n));
    k_ms_init<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, g->V, a->n, a->off, a->ea, a->eb, a->ew, a->bits);
    PG_LAUNCHED(ctx);
    if (a->M >= 2 && a->attempts > 0) {
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeCooperative;
        attr.val.cooperative = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(a->grid);
        cfg.blockDim = dim3(MS_THREADS);
        cfg.stream = ctx->stream;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_ms_rounds, *a));
        PG_LAUNCHED(ctx);
    }
    return PG_OK;
}

pg_status ms_rows_enqueue(pg_ctx* ctx, const pg_graph* g, MsArgs* a, int32_t* C_out, float* V_out)
{
    const int grid = ctx->sm_count * 4;
    k_ms_cursor<<<grid, 256, 0, ctx->stream>>>(g->R, a->n, a->cursor);
    PG_LAUNCHED(ctx);
    k_ms_scatter<<<grid, 256, 0, ctx->stream>>>(a->ea, a->eb, a->ew, a->M, a->cursor, a->ct, V_out ? a->vt : nullptr);
    PG_LAUNCHED(ctx);
    return launch_row_sort(ctx, g->R, a->n, a->ct, V_out ? a->vt : nullptr, C_out, V_out);
}

extern "C" int64_t pg_maslov_round_size(int64_t M) { return ms_round_size(M); }

extern "C" pg_status pg_maslov(pg_ctx* ctx, const pg_graph* g, uint64_t seed, int64_t attempts, pg_graph** out,
                               int64_t* committed)
{
    if (!ctx || !g || !out || attempts < 0) return pg_fail(ctx, PG_ERR_INVALID, "pg_maslov: bad arguments");
    if (g->nnz / 2 > INT32_MAX) return pg_fail(ctx, PG_ERR_TOO_LARGE, "pg_maslov: too many edges");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    MsArgs a;
    PG_TRY(ms_prepare(ctx, g, seed, attempts, &a));
    PG_TRY(ms_enqueue(ctx, g, &a));
    pg_graph* r;
    PG_TRY(pg_graph_alloc(ctx, g->n, g->nnz, g->V != nullptr, &r));
    cudaError_t e = cudaMemcpyAsync(r->R, g->R, sizeof(int32_t) * ((size_t)g->n + 1), cudaMemcpyDeviceToDevice,
                                    ctx->stream);
    pg_status st = e == cudaSuccess ? ms_rows_enqueue(ctx, g, &a, r->C, r->V)
                                    : pg_fail(ctx, PG_ERR_CUDA, "pg_maslov: %s", cudaGetErrorString(e));
    if (st != PG_OK) {
        pg_graph_free(r);
        return st;
    }
    *out = r;
    if (committed) {
        MsControl c;
        PG_TRY(pg_d2h(ctx, &c, a.st, sizeof c));
        *committed = (int64_t)c.committed;
    }
    return PG_OK;
}
