// clustering.cu -- clustering coefficients.
//   binary: Cp (U/Cp/Cp/Cp.cpp:21-116) from exact per-node triangle counts;
//   Onnela: Cp_2 (W/Cp/Cp/Cp_2.cpp:23-130).
//
// One CTA per node u (grid-stride).  The neighbour set of u is marked in a
// shared-memory bitmap of the node range (n bits), so every membership test
// of a neighbour's neighbour is one shared-memory load; the neighbour lists
// themselves are read coalesced, one warp per neighbour.  Binary counting
// only visits neighbours v > u and credits the pair count to both u and v,
// which halves the work (each triangle is then counted twice at each of its
// three nodes).
#include "pg_internal.cuh"
#include "clustering.cuh"
#include <cuda.h>
#include <algorithm>
#include <cmath>

namespace {
constexpr int THREADS = 256;

__global__ void __launch_bounds__(THREADS)
k_triangles(const int32_t* __restrict__ R, const int32_t* __restrict__ C, int32_t n,
            unsigned long long* __restrict__ tri2, int* __restrict__ next_node)
{
    extern __shared__ unsigned int bm[];
    __shared__ int s_u;
    __shared__ unsigned long long s_acc[THREADS / 32];
    const int W = (n + 31) >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = THREADS / 32;
    for (int w = threadIdx.x; w < W; w += THREADS) bm[w] = 0u;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_u = atomicAdd(next_node, 1);
        __syncthreads();
        const int u = s_u;
        if (u >= n) break;
        const int32_t s = R[u], e = R[u + 1];
        if (e - s < 2) continue;
        for (int32_t q = s + threadIdx.x; q < e; q += THREADS) atomicOr(&bm[C[q] >> 5], 1u << (C[q] & 31));
        __syncthreads();
        // first neighbour index with v > u (columns ascend)
        int32_t lo = s, hi = e;
        while (lo < hi) {
            int32_t mid = (lo + hi) >> 1;
            if (C[mid] > u) hi = mid; else lo = mid + 1;
        }
        unsigned long long acc_u = 0;
        for (int32_t q = lo + warp; q < e; q += nwarp) {
            const int v = C[q];
            unsigned int c = 0;
            for (int32_t f = R[v] + lane; f < R[v + 1]; f += 32) {
                int w = C[f];
                c += (bm[w >> 5] >> (w & 31)) & 1u;
            }
            c = __reduce_add_sync(0xffffffffu, c);
            if (lane == 0 && c) {
                atomicAdd(&tri2[v], (unsigned long long)c);
                acc_u += c;
            }
        }
        if (lane == 0) s_acc[warp] = acc_u;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < nwarp; w++) t += s_acc[w];
            if (t) atomicAdd(&tri2[u], t);
        }
        for (int32_t q = s + threadIdx.x; q < e; q += THREADS) bm[C[q] >> 5] = 0u;
    }
}

// Cp[k] = (double)t / k / (k-1) * 2 rounded to float (Cp.cpp:110), 0 for k < 2.
__global__ void k_cp_binary(const int32_t* __restrict__ R, int32_t n, const unsigned long long* __restrict__ tri2,
                            float* __restrict__ cp, long long* __restrict__ tri)
{
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        int k = R[u + 1] - R[u];
        unsigned long long t = tri2[u] >> 1;
        float c = 0.0f;
        if (k >= 2) {
            double x = (double)t;
            x = __ddiv_rn(x, (double)k);
            x = __ddiv_rn(x, (double)(k - 1));
            x = __dmul_rn(x, 2.0);
            c = __double2float_rn(x);
        }
        cp[u] = c;
        if (tri) tri[u] = (long long)t;
    }
}

// Deterministic FP64 mean of a float vector: one block, fixed order.
__global__ void k_mean_f32(const float* __restrict__ x, int32_t n, double* __restrict__ out)
{
    __shared__ double sh[1024];
    double a = 0.0;
    int per = (n + blockDim.x - 1) / blockDim.x;
    int lo = threadIdx.x * per, hi = min(n, lo + per);
    for (int i = lo; i < hi; i++) a += (double)x[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)blockDim.x; i++) t += sh[i];
        *out = n > 0 ? t / n : 0.0;
    }
}

// ---------------------------------------------------------------- Onnela
// A batch of graphs described by a table; a single graph is a table of one.
struct GraphRef {
    const int32_t* R;
    const int32_t* C;
    const float* V;
    int32_t n;
    int32_t node0;      // offset of this graph's nodes in the concatenated outputs
};

// vmax per graph: max over V[0..lim) (lim = n for the reference CPU rule,
// nnz otherwise).
__global__ void k_vmax(const GraphRef* __restrict__ gs, int ng, int first_n, float* __restrict__ vmax)
{
    for (int gi = blockIdx.x; gi < ng; gi += gridDim.x) {
        GraphRef g = gs[gi];
        long long nnz = g.R[g.n];
        long long lim = first_n ? min((long long)g.n, nnz) : nnz;
        float m = -INFINITY;
        for (long long q = threadIdx.x; q < lim; q += blockDim.x) m = fmaxf(m, g.V[q]);
        for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        __shared__ float sm[32];
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = -INFINITY;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmaxf(t, sm[w]);
            vmax[gi] = t;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int graph_of(const int* __restrict__ node0, int ng, int x)
{
    int lo = 0, hi = ng - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (node0[mid] <= x) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per node u: sum over connected neighbour pairs j < h of
// (w_jh w_uj w_uh)^(1/3), w = V / vmax (float division as Cp_2.cpp:37).
// The weight of (u, h) is found by binary search in u's sorted row.
__global__ void __launch_bounds__(THREADS)
k_onnela(const GraphRef* __restrict__ gs, const int* __restrict__ node0, int ng, int total_nodes,
         const float* __restrict__ vmax, float* __restrict__ cp, int* __restrict__ next_node)
{
    extern __shared__ unsigned int bm[];
    __shared__ int s_x;
    __shared__ double s_acc[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = THREADS / 32;
    int cur_g = -1;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_x = atomicAdd(next_node, 1);
        __syncthreads();
        const int x = s_x;
        if (x >= total_nodes) break;
        const int gi = graph_of(node0, ng, x);
        const GraphRef g = gs[gi];
        const int u = x - g.node0;
        const int W = (g.n + 31) >> 5;
        if (gi != cur_g) {
            for (int w = threadIdx.x; w < W; w += THREADS) bm[w] = 0u;
            cur_g = gi;
            __syncthreads();
        }
        const int32_t s = g.R[u], e = g.R[u + 1];
        const int k = e - s;
        if (k < 2) {
            if (threadIdx.x == 0) cp[x] = 0.0f;
            continue;
        }
        const float vm = vmax[gi];
        for (int32_t q = s + threadIdx.x; q < e; q += THREADS) atomicOr(&bm[g.C[q] >> 5], 1u << (g.C[q] & 31));
        __syncthreads();
        double acc = 0.0;
        for (int32_t q = s + warp; q < e; q += nwarp) {
            const int j = g.C[q];
            const double wuj = (double)__fdiv_rn(g.V[q], vm);
            for (int32_t f = g.R[j] + lane; f < g.R[j + 1]; f += 32) {
                const int h = g.C[f];
                if (h <= j || !((bm[h >> 5] >> (h & 31)) & 1u)) continue;
                const float wjh = __fdiv_rn(g.V[f], vm);
                if (wjh == 0.0f) continue;
                int32_t lo = s, hi = e - 1;
                while (lo < hi) {
                    int32_t mid = (lo + hi) >> 1;
                    if (g.C[mid] < h) lo = mid + 1; else hi = mid;
                }
                const double wuh = (double)__fdiv_rn(g.V[lo], vm);
                acc += pow((double)wjh * wuj * wuh, 1.0 / 3.0);
            }
        }
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) s_acc[warp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < nwarp; w++) t += s_acc[w];
            cp[x] = (float)(2.0 * t / k / (k - 1));
        }
        for (int32_t q = s + threadIdx.x; q < e; q += THREADS) bm[g.C[q] >> 5] = 0u;
    }
}

__global__ void k_mean_segments(const float* __restrict__ x, const int* __restrict__ node0, int ng, int total,
                                double* __restrict__ out)
{
    for (int gi = blockIdx.x; gi < ng; gi += gridDim.x) {
        if (threadIdx.x != 0) continue;
        int lo = node0[gi], hi = gi + 1 < ng ? node0[gi + 1] : total;
        double t = 0.0;
        for (int i = lo; i < hi; i++) t += (double)x[i];
        out[gi] = hi > lo ? t / (hi - lo) : 0.0;
    }
}
}  // namespace

// Onnela for a table of graphs already on the device (used by pg_fw_batched
// too): the table is uploaded (and the stream synchronised) here, the
// kernels are enqueued by onnela_enqueue.
pg_status onnela_prepare(pg_ctx* ctx, const pg_graph* const* graphs, int ng, int first_n, float* cp_dev,
                         double* mean_dev, OnnelaArgs* a)
{
    std::vector<GraphRef> tab(ng);
    std::vector<int> node0(ng);
    int total = 0, nmax = 1;
    for (int i = 0; i < ng; i++) {
        if (!graphs[i]->V) return pg_fail(ctx, PG_ERR_INVALID, "Onnela clustering needs a weighted graph");
        tab[i] = {graphs[i]->R, graphs[i]->C, graphs[i]->V, graphs[i]->n, total};
        node0[i] = total;
        total += graphs[i]->n;
        nmax = std::max(nmax, (int)graphs[i]->n);
    }
    GraphRef* dtab;
    PG_TRY(pg_wst(ctx, "on.tab", (size_t)ng, &dtab));
    PG_TRY(pg_wst(ctx, "on.node0", (size_t)ng, &a->node0));
    PG_TRY(pg_wst(ctx, "on.ctr", 1, &a->counter));
    PG_TRY(pg_wst(ctx, "on.vmax", (size_t)ng, &a->vmax));
    PG_CUDA(ctx, cudaMemcpyAsync(dtab, tab.data(), sizeof(GraphRef) * ng, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemcpyAsync(a->node0, node0.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, ctx->stream));
    a->smem = (size_t)((nmax + 31) / 32) * 4;
    if (a->smem > ctx->smem_optin - 4096) return pg_fail(ctx, PG_ERR_TOO_LARGE, "Onnela: n=%d too large", nmax);
    if (a->smem > 48 * 1024)
        PG_CUDA(ctx, cudaFuncSetAttribute(k_onnela, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a->smem));
    a->tab = dtab;
    a->ng = ng;
    a->total = total;
    a->first_n = first_n;
    a->cp = cp_dev;
    a->mean = mean_dev;
    // keep the host tables alive until the copies have been consumed
    PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return PG_OK;
}

pg_status onnela_enqueue(pg_ctx* ctx, const OnnelaArgs* a)
{
    const GraphRef* tab = (const GraphRef*)a->tab;
    PG_CUDA(ctx, cudaMemsetAsync(a->counter, 0, sizeof(int), ctx->stream));
    k_vmax<<<std::min(a->ng, 4096), 256, 0, ctx->stream>>>(tab, a->ng, a->first_n, a->vmax);
    PG_LAUNCHED(ctx);
    k_onnela<<<ctx->sm_count * 4, THREADS, a->smem, ctx->stream>>>(tab, a->node0, a->ng, a->total, a->vmax, a->cp,
                                                                   a->counter);
    PG_LAUNCHED(ctx);
    k_mean_segments<<<std::min(a->ng, 4096), 32, 0, ctx->stream>>>(a->cp, a->node0, a->ng, a->total, a->mean);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

pg_status pg_onnela_table(pg_ctx* ctx, const pg_graph* const* graphs, int ng, int first_n, float* cp_dev,
                          double* mean_dev)
{
    OnnelaArgs a;
    PG_TRY(onnela_prepare(ctx, graphs, ng, first_n, cp_dev, mean_dev, &a));
    return onnela_enqueue(ctx, &a);
}

// Binary clustering of one graph, enqueued only: per-node Cp (float), exact
// triangles (optional) and the FP64 mean over all nodes, in device memory.
pg_status binary_cp_prepare(pg_ctx* ctx, int n, BinaryCpArgs* a)
{
    PG_TRY(pg_wst(ctx, "cl.tri2", (size_t)n + 1, &a->tri2));
    PG_TRY(pg_wst(ctx, "cl.ctr", 1, &a->counter));
    a->smem = (size_t)((n + 31) / 32) * 4;
    if (a->smem > ctx->smem_optin - 4096) return pg_fail(ctx, PG_ERR_TOO_LARGE, "clustering: n=%d too large", n);
    if (a->smem > 48 * 1024)
        PG_CUDA(ctx, cudaFuncSetAttribute(k_triangles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a->smem));
    return PG_OK;
}

pg_status binary_cp_enqueue(pg_ctx* ctx, const BinaryCpArgs* a, const int32_t* R, const int32_t* C, int n, float* cp,
                            long long* tri, double* mean)
{
    PG_CUDA(ctx, cudaMemsetAsync(a->tri2, 0, sizeof(unsigned long long) * (n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(a->counter, 0, sizeof(int), ctx->stream));
    if (n > 0) {
        k_triangles<<<ctx->sm_count * 4, THREADS, a->smem, ctx->stream>>>(R, C, n, a->tri2, a->counter);
        PG_LAUNCHED(ctx);
        k_cp_binary<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(R, n, a->tri2, cp, tri);
        PG_LAUNCHED(ctx);
    }
    k_mean_f32<<<1, 1024, 0, ctx->stream>>>(cp, n, mean);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

extern "C" pg_status pg_clustering(pg_ctx* ctx, const pg_graph* g, int32_t kind, int32_t flags, float* cp,
                                   int64_t* triangles, double* mean)
{
    if (!ctx || !g || !cp) return pg_fail(ctx, PG_ERR_INVALID, "pg_clustering: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    float* dcp;
    double* dmean;
    PG_TRY(pg_wst(ctx, "cl.cp", (size_t)n + 1, &dcp));
    PG_TRY(pg_wst(ctx, "cl.mean", 1, &dmean));
    if (kind == 0) {
        long long* tri = nullptr;
        BinaryCpArgs a;
        PG_TRY(binary_cp_prepare(ctx, n, &a));
        if (triangles) PG_TRY(pg_wst(ctx, "cl.tri", (size_t)n + 1, &tri));
        PG_TRY(binary_cp_enqueue(ctx, &a, g->R, g->C, n, dcp, tri, dmean));
        if (triangles) PG_TRY(pg_d2h(ctx, triangles, tri, sizeof(long long) * n));
    } else if (kind == 1) {
        const pg_graph* one[1] = {g};
        PG_TRY(pg_onnela_table(ctx, one, 1, flags & 1, dcp, dmean));
    } else {
        return pg_fail(ctx, PG_ERR_INVALID, "unknown clustering kind %d", kind);
    }
    PG_TRY(pg_d2h(ctx, cp, dcp, sizeof(float) * n));
    if (mean) PG_TRY(pg_d2h(ctx, mean, dmean, sizeof(double)));
    return PG_OK;
}

// ------------------------------------------------ allocation-free variant
// Binary clustering for callers that cannot allocate device memory: host
// processes whose device memory is owned by someone else (a framework's
// caching allocator or a plugin host that reserves the GPU up front), and
// latency-critical pipelines that forbid cudaMalloc after start-up because
// it can synchronise the device.  The per-node triangle counters live in
// this file-scope device array instead of a workspace allocation.  Every
// call shares it and it keeps the last call's contents, so it is cleared at
// the start of each call, and calls that overlap on the GPU (other streams,
// other host threads) race on it.
namespace {
constexpr int64_t NOALLOC_SCRATCH_WORDS = (16LL << 20) / 8;   // 16 MiB: n + 2 counters
static __device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr int NOALLOC_SMEM_SLACK = 4096;   // static shared memory of k_triangles and margin

// Set-up state per device, filled by the first call with that device
// current: the array's device address (the host-side symbol is only a
// stand-in), the SM count and the opt-in shared memory per block, and the id
// of the CUDA context they belong to.  A new context on the device (after
// cudaDeviceReset) has a new id, and the next call resolves the address again.
struct NoallocDevice {
    unsigned long long* scratch;
    unsigned long long ctx_id;
    int sm_count;
    int smem_optin;
};
static NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

__global__ void k_noalloc_clear(unsigned long long* __restrict__ w, int64_t count)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < count; q += (int64_t)gridDim.x * blockDim.x)
        w[q] = 0ULL;
}

// Largest n whose neighbour bitmap (n bits) fits the opt-in shared memory.
int64_t noalloc_smem_nodes(int smem_optin) { return (int64_t)(smem_optin - NOALLOC_SMEM_SLACK) / 4 * 32; }

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points
// (the library does not link the driver library directly).
bool current_ctx_id(unsigned long long* id)
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) != cudaSuccess ||
            r1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) != cudaSuccess ||
            r2 != cudaDriverEntryPointSuccess)
            return false;
        get_current = (GetCurrent)p;
        get_id = (GetId)q;
    }
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) return false;
    return get_id(c, id) == CUDA_SUCCESS;
}

pg_status noalloc_setup(int dev, NoallocDevice** out)
{
    NoallocDevice& d = g_noalloc_dev[dev];
    unsigned long long id = 0;
    if (d.scratch && current_ctx_id(&id) && id == d.ctx_id) {
        *out = &d;
        return PG_OK;
    }
    void* p = nullptr;   // resolving the symbol also initialises the device's context
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PG_ERR_CUDA;
    int sms = 0, optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return PG_ERR_CUDA;
    if (!current_ctx_id(&id)) return PG_ERR_CUDA;
    d.scratch = (unsigned long long*)p;
    d.ctx_id = id;
    d.sm_count = sms;
    d.smem_optin = optin;
    *out = &d;
    return PG_OK;
}
}  // namespace

extern "C" int64_t pg_clustering_noalloc_max_nodes(void)
{
    int64_t lim = NOALLOC_SCRATCH_WORDS - 2;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess)
        lim = std::min(lim, noalloc_smem_nodes(optin));
    return lim;
}

extern "C" pg_status pg_clustering_noalloc(const int32_t* R, const int32_t* C, int32_t n, float* cp, int64_t* triangles,
                                           void* stream)
{
    if (!R || !cp || n < 0) return PG_ERR_INVALID;
    if ((int64_t)n > NOALLOC_SCRATCH_WORDS - 2) return PG_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PG_ERR_NO_DEVICE;
    NoallocDevice* d = nullptr;
    if (pg_status st = noalloc_setup(dev, &d); st != PG_OK) return st;
    if (n == 0) return PG_OK;
    if ((int64_t)n > noalloc_smem_nodes(d->smem_optin)) return PG_ERR_TOO_LARGE;
    const size_t smem = (size_t)((n + 31) / 32) * 4;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_triangles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PG_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* tri2 = d->scratch;
    int* next_node = (int*)(tri2 + (n + 1));
    k_noalloc_clear<<<d->sm_count, 256, 0, st>>>(tri2, (int64_t)n + 2);
    k_triangles<<<d->sm_count * 4, THREADS, smem, st>>>(R, C, n, tri2, next_node);
    k_cp_binary<<<d->sm_count * 4, 256, 0, st>>>(R, n, tri2, cp, (long long*)triangles);
    return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_CUDA;
}
