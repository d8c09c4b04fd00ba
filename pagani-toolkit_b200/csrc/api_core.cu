// api_core.cu -- context, errors, workspace, graph objects, CSR assembly,
// degree and the small host-side ratios of the C ABI.
#include "pg_internal.cuh"
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <new>

// ------------------------------------------------------------------ errors
pg_status pg_fail(pg_ctx* ctx, pg_status s, const char* fmt, ...)
{
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return s;
}

extern "C" const char* pg_last_error(const pg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" const char* pg_status_string(pg_status s)
{
    switch (s) {
    case PG_OK: return "ok";
    case PG_ERR_INVALID: return "invalid argument";
    case PG_ERR_CUDA: return "CUDA error";
    case PG_ERR_NOMEM: return "out of device memory";
    case PG_ERR_TOO_LARGE: return "result too large for the CSR format";
    case PG_ERR_INTERNAL: return "internal check failed";
    case PG_ERR_TIMEOUT: return "bounded device wait timed out";
    case PG_ERR_NO_DEVICE: return "no usable sm_100 device";
    }
    return "unknown status";
}

// ----------------------------------------------------------------- context
extern "C" pg_status pg_create(pg_ctx** out, int device)
{
    if (!out) return PG_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return PG_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return PG_ERR_INVALID;
    pg_ctx* ctx = new (std::nothrow) pg_ctx;
    if (!ctx) return PG_ERR_NOMEM;
    ctx->device = device;
    cudaDeviceProp prop;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete ctx;
        return PG_ERR_NO_DEVICE;
    }
    if (prop.major < 10) {  // the library carries sm_100a code only
        delete ctx;
        return PG_ERR_NO_DEVICE;
    }
    ctx->sm_count = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return PG_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    // graphs come from the device's stream-ordered pool; keeping freed
    // blocks in the pool makes the per-subject graph allocation cheap
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = ctx;
    return PG_OK;
}

extern "C" pg_status pg_destroy(pg_ctx* ctx)
{
    if (!ctx) return PG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->ws) cudaFree(kv.second.p);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    for (auto& kv : ctx->hws) cudaFreeHost(kv.second.p);
    for (auto& st : ctx->pool) cudaStreamDestroy(st);
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    for (auto& sp : ctx->prof_open) {
        cudaEventDestroy(sp.a);
        cudaEventDestroy(sp.b);
    }
    for (auto& e : ctx->prof_free) cudaEventDestroy(e);
    for (auto& st : ctx->side)
        if (st) cudaStreamDestroy(st);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PG_OK;
}

extern "C" pg_status pg_synchronize(pg_ctx* ctx)
{
    if (!ctx) return PG_ERR_INVALID;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

extern "C" void* pg_stream(pg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

// ---------------------------------------------------------------- profiling
static cudaEvent_t prof_event(pg_ctx* ctx)
{
    if (!ctx->prof_free.empty()) {
        cudaEvent_t e = ctx->prof_free.back();
        ctx->prof_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

int pg_prof_begin(pg_ctx* ctx, const char* name)
{
    if (!ctx->prof) return -1;
    cudaEvent_t a = prof_event(ctx), b = prof_event(ctx);
    if (!a || !b) return -1;
    cudaEventRecord(a, ctx->stream);
    ctx->prof_open.push_back({name, a, b});
    return (int)ctx->prof_open.size() - 1;
}

void pg_prof_end(pg_ctx* ctx, int handle)
{
    if (handle < 0 || handle >= (int)ctx->prof_open.size()) return;
    cudaEventRecord(ctx->prof_open[handle].b, ctx->stream);
}

// Folds the recorded spans into the per-kernel sums (synchronises the stream).
static pg_status prof_resolve(pg_ctx* ctx)
{
    if (ctx->prof_open.empty()) return PG_OK;
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (auto& sp : ctx->prof_open) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) {
            auto& acc = ctx->prof_sum[sp.name];
            acc.first++;
            acc.second += ms;
        } else {
            cudaGetLastError();
        }
        ctx->prof_free.push_back(sp.a);
        ctx->prof_free.push_back(sp.b);
    }
    ctx->prof_open.clear();
    return PG_OK;
}

extern "C" pg_status pg_profile_enable(pg_ctx* ctx, int32_t on)
{
    if (!ctx) return PG_ERR_INVALID;
    PG_TRY(prof_resolve(ctx));
    ctx->prof = on != 0;
    return PG_OK;
}

extern "C" pg_status pg_profile_reset(pg_ctx* ctx)
{
    if (!ctx) return PG_ERR_INVALID;
    PG_TRY(prof_resolve(ctx));
    ctx->prof_sum.clear();
    return PG_OK;
}

extern "C" pg_status pg_profile_get(pg_ctx* ctx, const char* kernel, int64_t* launches, double* ms)
{
    if (!ctx || !kernel) return pg_fail(ctx, PG_ERR_INVALID, "pg_profile_get: null argument");
    PG_TRY(prof_resolve(ctx));
    auto it = ctx->prof_sum.find(kernel);
    if (launches) *launches = it == ctx->prof_sum.end() ? 0 : it->second.first;
    if (ms) *ms = it == ctx->prof_sum.end() ? 0.0 : it->second.second;
    return PG_OK;
}
extern "C" int64_t pg_launch_count(const pg_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" pg_status pg_debug_stall_next_gram(pg_ctx* ctx, uint64_t wait_ns)
{
    if (!ctx) return PG_ERR_INVALID;
    ctx->debug_gram_stall_ns = wait_ns;
    return PG_OK;
}

// --------------------------------------------------------------- workspace
pg_status pg_ws(pg_ctx* ctx, const char* key, size_t bytes, void** out)
{
    auto& b = ctx->ws[key];
    if (b.bytes < bytes) {
        if (b.p) {
            PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(b.p);
            b.p = nullptr;
            b.bytes = 0;
        }
        size_t want = bytes + bytes / 8;  // head room for slowly growing sizes
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return pg_fail(ctx, PG_ERR_NOMEM, "workspace '%s': cannot allocate %zu bytes", key, want);
        }
        b.bytes = want;
    }
    *out = b.p;
    return PG_OK;
}

pg_status pg_pinned(pg_ctx* ctx, size_t bytes, void** out)
{
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        PG_CUDA(ctx, cudaMallocHost(&ctx->pinned, bytes));
        ctx->pinned_bytes = bytes;
    }
    *out = ctx->pinned;
    return PG_OK;
}

pg_status pg_hws(pg_ctx* ctx, const char* key, size_t bytes, void** out)
{
    auto& b = ctx->hws[key];
    if (b.bytes < bytes) {
        if (b.p) {
            PG_CUDA(ctx, cudaDeviceSynchronize());
            cudaFreeHost(b.p);
            b.p = nullptr;
            b.bytes = 0;
        }
        const size_t want = bytes + bytes / 8;
        if (cudaMallocHost(&b.p, want) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return pg_fail(ctx, PG_ERR_NOMEM, "pinned buffer '%s': cannot allocate %zu bytes", key, want);
        }
        b.bytes = want;
    }
    *out = b.p;
    return PG_OK;
}

pg_status pg_stream_pool(pg_ctx* ctx, size_t count)
{
    while (ctx->pool.size() < count) {
        cudaStream_t st;
        PG_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        ctx->pool.push_back(st);
    }
    return PG_OK;
}

pg_status pg_d2h(pg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (!bytes) return PG_OK;
    PG_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

pg_status pg_h2d(pg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (!bytes) return PG_OK;
    PG_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

// ------------------------------------------------------------------ graphs
pg_status pg_graph_alloc(pg_ctx* ctx, int32_t n, int64_t nnz, bool weighted, pg_graph** out)
{
    pg_graph* g = new (std::nothrow) pg_graph;
    if (!g) return PG_ERR_NOMEM;
    g->ctx = ctx;
    g->device = ctx->device;
    g->n = n;
    g->nnz = nnz;
    // stream-ordered on the context stream (pg_graph_free's cudaFree waits for
    // the device before the blocks return to the pool)
    cudaError_t e = cudaMallocAsync((void**)&g->R, sizeof(int32_t) * ((size_t)n + 1), ctx->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&g->C, sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1), ctx->stream);
    if (e == cudaSuccess && weighted)
        e = cudaMallocAsync((void**)&g->V, sizeof(float) * (size_t)(nnz > 0 ? nnz : 1), ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(g->R); cudaFree(g->C); cudaFree(g->V);
        delete g;
        return pg_fail(ctx, PG_ERR_NOMEM, "graph allocation (n=%d nnz=%lld) failed", n, (long long)nnz);
    }
    *out = g;
    return PG_OK;
}

extern "C" pg_status pg_graph_free(pg_graph* g)
{
    if (!g) return PG_OK;
    // cudaFree waits for the device work that may still use the arrays; the
    // graph does not touch its creating context, which may already be gone.
    cudaSetDevice(g->device);
    cudaFree(g->R);
    cudaFree(g->C);
    cudaFree(g->V);
    delete g;
    return PG_OK;
}

extern "C" pg_status pg_graph_info(const pg_graph* g, int32_t* n, int64_t* nnz, int32_t* weighted)
{
    if (!g) return PG_ERR_INVALID;
    if (n) *n = g->n;
    if (nnz) *nnz = g->nnz;
    if (weighted) *weighted = g->V != nullptr;
    return PG_OK;
}

extern "C" pg_status pg_graph_from_csr(pg_ctx* ctx, const int32_t* R, const int32_t* C, const float* V,
                                       int32_t n, int64_t nnz, int32_t on_device, pg_graph** out)
{
    if (!ctx || !out || !R || (nnz > 0 && !C) || n < 0 || nnz < 0)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_graph_from_csr: bad arguments");
    if (nnz > INT32_MAX) return pg_fail(ctx, PG_ERR_TOO_LARGE, "nnz %lld exceeds int32", (long long)nnz);
    if (!on_device && (int64_t)R[n] != nnz)
        return pg_fail(ctx, PG_ERR_INVALID, "R[n]=%d does not match nnz=%lld", R[n], (long long)nnz);
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    pg_graph* g;
    PG_TRY(pg_graph_alloc(ctx, n, nnz, V != nullptr, &g));
    cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = cudaMemcpyAsync(g->R, R, sizeof(int32_t) * ((size_t)n + 1), k, ctx->stream);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(g->C, C, sizeof(int32_t) * (size_t)nnz, k, ctx->stream);
    if (e == cudaSuccess && V && nnz) e = cudaMemcpyAsync(g->V, V, sizeof(float) * (size_t)nnz, k, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        pg_graph_free(g);
        return pg_fail(ctx, PG_ERR_CUDA, "pg_graph_from_csr copy: %s", cudaGetErrorString(e));
    }
    *out = g;
    return PG_OK;
}

extern "C" pg_status pg_graph_to_csr(pg_ctx* ctx, const pg_graph* g, int32_t* R, int32_t* C, float* V,
                                     int32_t on_device)
{
    if (!ctx || !g) return pg_fail(ctx, PG_ERR_INVALID, "pg_graph_to_csr: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (R) PG_CUDA(ctx, cudaMemcpyAsync(R, g->R, sizeof(int32_t) * ((size_t)g->n + 1), k, ctx->stream));
    if (C && g->nnz) PG_CUDA(ctx, cudaMemcpyAsync(C, g->C, sizeof(int32_t) * (size_t)g->nnz, k, ctx->stream));
    if (V && g->V && g->nnz) PG_CUDA(ctx, cudaMemcpyAsync(V, g->V, sizeof(float) * (size_t)g->nnz, k, ctx->stream));
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

// ------------------------------------------------------------------- scan
// Exclusive scan of n int32 counts into n+1 int64 offsets, three phases over
// blocks of 1024 elements.
static constexpr int SCAN_B = 1024;

__device__ __forceinline__ long long block_excl_scan_1024(long long v, long long* sh, long long* total)
{
    // 1024 threads: warp scan, then scan of 32 warp totals.
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        long long t = sh[lane];
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        sh[lane] = t;
    }
    __syncthreads();
    long long incl = x + (w ? sh[w - 1] : 0);
    if (total) *total = sh[31];
    return incl - v;
}

__global__ void k_scan_blocks(const int32_t* __restrict__ cnt, int32_t n, long long* __restrict__ off,
                              long long* __restrict__ bsum)
{
    __shared__ long long sh[32];
    long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
    long long v = i < n ? cnt[i] : 0;
    long long tot;
    long long ex = block_excl_scan_1024(v, sh, &tot);
    if (i < n) off[i] = ex;
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_sums(long long* __restrict__ bsum, int nb, long long* __restrict__ total)
{
    __shared__ long long sh[32];
    long long carry = 0;
    for (int base = 0; base < nb; base += SCAN_B) {
        int i = base + threadIdx.x;
        long long v = i < nb ? bsum[i] : 0;
        long long tot;
        long long ex = block_excl_scan_1024(v, sh, &tot);
        __syncthreads();
        if (i < nb) bsum[i] = ex + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(long long* __restrict__ off, int32_t n, const long long* __restrict__ bsum,
                           const long long* __restrict__ total)
{
    long long i = (long long)blockIdx.x * SCAN_B + threadIdx.x;
    if (i < n) off[i] += bsum[blockIdx.x];
    if (i == 0) off[n] = *total;
}

pg_status pg_scan_counts(pg_ctx* ctx, const int32_t* cnt, int64_t* off, int32_t n)
{
    int nb = ceil_div(n > 0 ? n : 1, SCAN_B);
    long long* bsum;
    PG_TRY(pg_wst(ctx, "scan.bsum", (size_t)nb + 1, &bsum));
    k_scan_blocks<<<nb, SCAN_B, 0, ctx->stream>>>(cnt, n, (long long*)off, bsum);
    PG_LAUNCHED(ctx);
    k_scan_sums<<<1, SCAN_B, 0, ctx->stream>>>(bsum, nb, bsum + nb);
    PG_LAUNCHED(ctx);
    k_scan_add<<<nb, SCAN_B, 0, ctx->stream>>>((long long*)off, n, bsum, bsum + nb);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

// ------------------------------------------------------ pairs -> CSR
__global__ void k_pair_degrees(const int2* __restrict__ pairs, long long np, int32_t* __restrict__ cnt)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int2 e = pairs[p];
        atomicAdd(&cnt[e.x], 1);
        atomicAdd(&cnt[e.y], 1);
    }
}

__global__ void k_off_to_rowptr(const long long* __restrict__ off, int32_t n, int32_t* __restrict__ R,
                                int32_t* __restrict__ cursor)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= n;
         i += (long long)gridDim.x * blockDim.x) {
        R[i] = (int32_t)off[i];
        if (i < n) cursor[i] = (int32_t)off[i];
    }
}

__global__ void k_pair_scatter(const int2* __restrict__ pairs, const float* __restrict__ w, long long np,
                               int32_t* __restrict__ cursor, int32_t* __restrict__ C, float* __restrict__ V)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int2 e = pairs[p];
        int32_t a = atomicAdd(&cursor[e.x], 1);
        int32_t b = atomicAdd(&cursor[e.y], 1);
        C[a] = e.y;
        C[b] = e.x;
        if (V) {
            float x = w[p];
            V[a] = x;
            V[b] = x;
        }
    }
}

// Per-row sort through a shared-memory bitmap of the column range: set one
// bit per entry, then every thread owns a run of words; an entry's rank is
// the popcount of the bits below it.  Out of place (Cin/Vin -> Cout/Vout).
__global__ void k_row_bitmap_sort(const int32_t* __restrict__ R, int32_t n, const int32_t* __restrict__ Cin,
                                  const float* __restrict__ Vin, int32_t* __restrict__ Cout,
                                  float* __restrict__ Vout)
{
    extern __shared__ unsigned int bm[];
    __shared__ int base[1024];
    const int W = (n + 31) >> 5;
    const int B = blockDim.x;
    const int cw = (W + B - 1) / B;
    for (int row = blockIdx.x; row < n; row += gridDim.x) {
        int32_t s = R[row], e = R[row + 1];
        if (e - s <= 1) {
            if (e - s == 1 && threadIdx.x == 0) {
                Cout[s] = Cin[s];
                if (Vin) Vout[s] = Vin[s];
            }
            continue;
        }
        for (int w = threadIdx.x; w < W; w += B) bm[w] = 0u;
        __syncthreads();
        for (int32_t q = s + threadIdx.x; q < e; q += B) {
            int c = Cin[q];
            atomicOr(&bm[c >> 5], 1u << (c & 31));
        }
        __syncthreads();
        int w0 = threadIdx.x * cw, w1 = min(W, w0 + cw);
        int cntb = 0;
        for (int w = w0; w < w1; w++) cntb += __popc(bm[w]);
        base[threadIdx.x] = cntb;
        __syncthreads();
        // exclusive scan of base[] (B <= 1024) by one warp
        if (threadIdx.x < 32) {
            int per = (B + 31) / 32;
            int lo = threadIdx.x * per, hi = min(B, lo + per);
            int acc = 0;
            for (int q = lo; q < hi; q++) acc += base[q];
            int x = acc;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (threadIdx.x >= o) x += y;
            }
            int run = x - acc;
            for (int q = lo; q < hi; q++) {
                int t = base[q];
                base[q] = run;
                run += t;
            }
        }
        __syncthreads();
        if (!Vin) {
            int pos = s + base[threadIdx.x];
            for (int w = w0; w < w1; w++) {
                unsigned m = bm[w];
                while (m) {
                    int b = __ffs(m) - 1;
                    m &= m - 1;
                    Cout[pos++] = (w << 5) | b;
                }
            }
        } else {
            for (int32_t q = s + threadIdx.x; q < e; q += B) {
                int c = Cin[q];
                int w = c >> 5;
                int owner = w / cw;
                int r = base[owner];
                for (int x = owner * cw; x < w; x++) r += __popc(bm[x]);
                r += __popc(bm[w] & ((1u << (c & 31)) - 1u));
                Cout[s + r] = c;
                Vout[s + r] = Vin[q];
            }
        }
        __syncthreads();
    }
}

pg_status launch_row_sort(pg_ctx* ctx, const int32_t* R, int32_t n, const int32_t* Cin,
                          const float* Vin, int32_t* Cout, float* Vout)
{
    // largest dynamic shared memory granted to the kernel so far, per device
    // (set once outside any stream capture, then only launches)
    static size_t granted[64];
    size_t smem = (size_t)((n + 31) / 32) * 4;
    if (smem > ctx->smem_optin - 8192)
        return pg_fail(ctx, PG_ERR_TOO_LARGE, "row sort: n=%d exceeds the shared-memory bitmap", n);
    if (smem > 48 * 1024 && (ctx->device >= 64 || smem > granted[ctx->device])) {
        PG_CUDA(ctx, cudaFuncSetAttribute(k_row_bitmap_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        if (ctx->device < 64) granted[ctx->device] = smem;
    }
    int grid = ctx->sm_count * 4;
    if (grid > n) grid = n > 0 ? n : 1;
    k_row_bitmap_sort<<<grid, 256, smem, ctx->stream>>>(R, n, Cin, Vin, Cout, Vout);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

pg_status pg_csr_sort_rows(pg_ctx* ctx, pg_graph* g)
{
    if (g->nnz == 0) return PG_OK;
    int32_t* Ct;
    float* Vt = nullptr;
    PG_TRY(pg_wst(ctx, "sort.C", (size_t)g->nnz, &Ct));
    if (g->V) PG_TRY(pg_wst(ctx, "sort.V", (size_t)g->nnz, &Vt));
    PG_CUDA(ctx, cudaMemcpyAsync(Ct, g->C, sizeof(int32_t) * g->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    if (g->V)
        PG_CUDA(ctx, cudaMemcpyAsync(Vt, g->V, sizeof(float) * g->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    return launch_row_sort(ctx, g->R, g->n, Ct, Vt, g->C, g->V);
}

pg_status pg_csr_from_pairs(pg_ctx* ctx, int32_t n, const int2* pairs, const float* w, int64_t npairs,
                            pg_graph** out)
{
    if (2 * npairs > INT32_MAX)
        return pg_fail(ctx, PG_ERR_TOO_LARGE, "%lld directed entries exceed the int32 CSR", 2LL * npairs);
    int32_t* cnt;
    long long* off;
    PG_TRY(pg_wst(ctx, "csr.cnt", (size_t)n + 1, &cnt));
    PG_TRY(pg_wst(ctx, "csr.off", (size_t)n + 2, &off));
    PG_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ((size_t)n + 1), ctx->stream));
    int grid = ctx->sm_count * 8;
    if (npairs > 0) {
        k_pair_degrees<<<grid, 256, 0, ctx->stream>>>(pairs, npairs, cnt);
        PG_LAUNCHED(ctx);
    }
    PG_TRY(pg_scan_counts(ctx, cnt, (int64_t*)off, n));
    pg_graph* g;
    PG_TRY(pg_graph_alloc(ctx, n, 2 * npairs, w != nullptr, &g));
    int32_t* cursor = cnt;  // counts are no longer needed
    k_off_to_rowptr<<<ceil_div((long long)n + 1, 256), 256, 0, ctx->stream>>>(off, n, g->R, cursor);
    PG_LAUNCHED(ctx);
    if (npairs > 0) {
        int32_t* Ct;
        float* Vt = nullptr;
        pg_status st = pg_wst(ctx, "sort.C", (size_t)(2 * npairs), &Ct);
        if (st == PG_OK && w) st = pg_wst(ctx, "sort.V", (size_t)(2 * npairs), &Vt);
        if (st != PG_OK) { pg_graph_free(g); return st; }
        k_pair_scatter<<<grid, 256, 0, ctx->stream>>>(pairs, w, npairs, cursor, Ct, Vt);
        ctx->launches++;
        st = launch_row_sort(ctx, g->R, n, Ct, Vt, g->C, g->V);
        if (st != PG_OK) { pg_graph_free(g); return st; }
    }
    *out = g;
    return PG_OK;
}

// ------------------------------------------------------------------ degree
// U/Degree/Degree/Degree.cpp:85-91: (float)R[k+1] - R[k];
// W/Degree/Degree/Degree.cpp:82-88: sequential float sum of V over the row.
__global__ void k_degree(const int32_t* __restrict__ R, const float* __restrict__ V, int32_t n,
                         float* __restrict__ deg, int* __restrict__ iso)
{
    int local = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int32_t s = R[k], e = R[k + 1];
        float d;
        if (V) {
            d = 0.0f;
            for (int32_t q = s; q < e; q++) d = __fadd_rn(d, V[q]);
        } else {
            d = __fsub_rn((float)e, (float)s);
        }
        deg[k] = d;
        local += (e == s);
    }
    local = __reduce_add_sync(0xffffffffu, local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(iso, local);
}

extern "C" pg_status pg_degree(pg_ctx* ctx, const pg_graph* g, float* deg, int32_t* isolated)
{
    if (!ctx || !g || !deg) return pg_fail(ctx, PG_ERR_INVALID, "pg_degree: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    float* d;
    int* iso;
    PG_TRY(pg_wst(ctx, "deg.out", (size_t)g->n + 1, &d));
    PG_TRY(pg_wst(ctx, "deg.iso", 1, &iso));
    PG_CUDA(ctx, cudaMemsetAsync(iso, 0, sizeof(int), ctx->stream));
    int grid = ctx->sm_count * 4;
    k_degree<<<grid, 256, 0, ctx->stream>>>(g->R, g->V, g->n, d, iso);
    PG_LAUNCHED(ctx);
    PG_TRY(pg_d2h(ctx, deg, d, sizeof(float) * (size_t)g->n));
    if (isolated) PG_TRY(pg_d2h(ctx, isolated, iso, sizeof(int)));
    return PG_OK;
}

// ----------------------------------------------------------- small-world
extern "C" pg_status pg_smallworld(double cp, const double* cp_rand, int32_t n_cp, double lp,
                                   const double* lp_rand, int32_t n_lp, double* gamma, double* lambda,
                                   double* sigma)
{
    double g = NAN, l = NAN;
    if (n_cp > 0 && cp_rand) {
        double s = 0;
        for (int i = 0; i < n_cp; i++) s += cp_rand[i];
        g = cp / (s / n_cp);
    }
    if (n_lp > 0 && lp_rand) {
        double s = 0;
        for (int i = 0; i < n_lp; i++) s += lp_rand[i];
        l = lp / (s / n_lp);
    }
    if (gamma) *gamma = g;
    if (lambda) *lambda = l;
    if (sigma) *sigma = g / l;
    return PG_OK;
}

// Reference: CorMat.cpp:310-312 (the long long product is converted to float
// and multiplied by the float sparsity before the double division).
extern "C" int64_t pg_sparsity_edges(int32_t N, float s)
{
    long long M1 = (long long)(N - 1) * N / 2;
    float prod = (float)(2LL * M1) * s;
    long long Clength = (long long)((double)prod / 100.0);
    Clength += Clength % 2;
    return Clength / 2;
}
