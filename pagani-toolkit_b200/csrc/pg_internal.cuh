// pg_internal.cuh -- context, graph and workspace types shared by the
// libpagani translation units, plus small device helpers.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <string>
#include <vector>
#include <map>
#include "../../include/pagani.h"

struct pg_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side[6] = {};  // created on first use; kernels that run beside `stream`
    cudaEvent_t ev[8] = {};
    int64_t launches = 0;
    std::string err;
    // Reusable device buffers keyed by name; grown on demand.
    struct Buf { void* p = nullptr; size_t bytes = 0; };
    std::map<std::string, Buf> ws;
    // Pinned host staging for small D2H/H2D transfers.
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // Pinned host buffers keyed by name, grown on demand, and a pool of
    // non-blocking streams: for host loops that keep many streams busy.
    std::map<std::string, Buf> hws;
    std::vector<cudaStream_t> pool;
    // Optional per-kernel device time (pg_profile_enable): event pairs around
    // the launches of named kernels, resolved when read.
    bool prof = false;
    struct ProfSpan { const char* name; cudaEvent_t a, b; };
    std::vector<ProfSpan> prof_open;
    std::map<std::string, std::pair<int64_t, double>> prof_sum;
    std::vector<cudaEvent_t> prof_free;
    // failure-path test hook (pg_debug_stall_next_gram): the next tcgen05 Gram
    // launch waits this long on a barrier nothing arrives on, then gives up
    unsigned long long debug_gram_stall_ns = 0;
};

struct pg_graph {
    pg_ctx* ctx = nullptr;  // creator; not used after pg_destroy
    int device = 0;
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t* R = nullptr;   // device
    int32_t* C = nullptr;   // device
    float* V = nullptr;     // device, may be null
};

// ---------------------------------------------------------------- errors
pg_status pg_fail(pg_ctx* ctx, pg_status s, const char* fmt, ...);

#define PG_CUDA(ctx, call)                                                              \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            return pg_fail((ctx), e_ == cudaErrorMemoryAllocation ? PG_ERR_NOMEM         \
                                                                  : PG_ERR_CUDA,        \
                           "%s:%d %s: %s", __FILE__, __LINE__, #call,                   \
                           cudaGetErrorString(e_));                                     \
        }                                                                               \
    } while (0)

#define PG_TRY(call)                        \
    do {                                    \
        pg_status s_ = (call);              \
        if (s_ != PG_OK) return s_;         \
    } while (0)

// Check the launch that was just issued and count it.
#define PG_LAUNCHED(ctx)                                                                \
    do {                                                                                \
        (ctx)->launches++;                                                              \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess)                                                          \
            return pg_fail((ctx), PG_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,   \
                           cudaGetErrorString(e_));                                     \
    } while (0)

// ------------------------------------------------------------- profiling
// With profiling on, pg_prof_begin records an event on the context stream
// before a launch of kernel `name` and returns a handle for pg_prof_end
// (after the launch); both are no-ops (handle -1) when profiling is off.
int pg_prof_begin(pg_ctx* ctx, const char* name);
void pg_prof_end(pg_ctx* ctx, int handle);

// ------------------------------------------------------------- workspace
// Device buffer named `key`, at least `bytes` long (contents undefined).
pg_status pg_ws(pg_ctx* ctx, const char* key, size_t bytes, void** out);
template <class T>
inline pg_status pg_wst(pg_ctx* ctx, const char* key, size_t count, T** out)
{
    return pg_ws(ctx, key, count * sizeof(T) + 256, (void**)out);
}
// Pinned host staging buffer of at least `bytes`.
pg_status pg_pinned(pg_ctx* ctx, size_t bytes, void** out);
// Pinned host buffer named `key`, at least `bytes` long (contents undefined;
// growing it synchronises the device).
pg_status pg_hws(pg_ctx* ctx, const char* key, size_t bytes, void** out);
template <class T>
inline pg_status pg_hwst(pg_ctx* ctx, const char* key, size_t count, T** out)
{
    return pg_hws(ctx, key, count * sizeof(T) + 256, (void**)out);
}
// At least `count` streams in ctx->pool.
pg_status pg_stream_pool(pg_ctx* ctx, size_t count);

// Copies between host and device on the context stream, synchronous.
pg_status pg_d2h(pg_ctx* ctx, void* dst, const void* src, size_t bytes);
pg_status pg_h2d(pg_ctx* ctx, void* dst, const void* src, size_t bytes);

// Creates a graph object that owns freshly allocated device arrays.
pg_status pg_graph_alloc(pg_ctx* ctx, int32_t n, int64_t nnz, bool weighted, pg_graph** out);

// CSR assembly from an unordered list of undirected pairs (i < j not
// required, i != j): degrees, exclusive scan, scatter, per-row sort.
// w may be null.  Result graph owns its arrays.
pg_status pg_csr_from_pairs(pg_ctx* ctx, int32_t n, const int2* pairs, const float* w,
                            int64_t npairs, pg_graph** out);
// Sorts the columns of every row ascending (carrying V when present).
pg_status pg_csr_sort_rows(pg_ctx* ctx, pg_graph* g);
// Row sort of a CSR whose rows are filled but unordered: Cin/Vin -> Cout/Vout
// (Vin may be null).  Only launches kernels (capture-safe once the kernel's
// shared-memory attribute has been set by a first call).
pg_status launch_row_sort(pg_ctx* ctx, const int32_t* R, int32_t n, const int32_t* Cin, const float* Vin,
                          int32_t* Cout, float* Vout);

// Exclusive scan of int32 counts into int64 offsets (n+1 entries).
pg_status pg_scan_counts(pg_ctx* ctx, const int32_t* cnt, int64_t* off, int32_t n);

// ------------------------------------------------------------- device
__device__ __forceinline__ int warp_lane() { return threadIdx.x & 31; }

// Order-preserving map from double to uint64 (larger double -> larger key).
__device__ __host__ __forceinline__ uint64_t dkey(double x)
{
    uint64_t u;
    memcpy(&u, &x, 8);
    return (u & 0x8000000000000000ULL) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __host__ __forceinline__ double dkey_inv(uint64_t k)
{
    uint64_t u = (k & 0x8000000000000000ULL) ? (k & ~0x8000000000000000ULL) : ~k;
    double x;
    memcpy(&x, &u, 8);
    return x;
}

// Warp-aggregated append: every lane with `want` gets a distinct slot.
// Returns the slot index or -1.  All lanes of the warp must call it.
__device__ __forceinline__ long long warp_append(unsigned long long* counter, bool want)
{
    unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return -1;
    int lane = warp_lane();
    int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!want) return -1;
    return (long long)(base + __popc(m & ((1u << lane) - 1)));
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
