// newman.cu -- Newman leading-eigenvector modularity (Partition_GPU /
// Sub_Partition_GPU / Lead_Vector_GPU, U/cuda_EC/cuda_EC/modularity_GPU.cu:230-530;
// CPU twins Partition / Sub_Partition / Lead_Vector, Modularity_CPU.cpp:48-298).
//
// The reference walks rounds r = 0, 1, ...: round r takes the nodes labelled
// r, finds the leading eigenvector of the generalised modularity matrix
// B(g) - diag(sumBG) by power iteration from v = node ids (tolerance 1e-6 on
// |v - v0| or |v + v0|, at most 10,000 iterations, rerun with a shift when
// the eigenvalue is negative) and, when lambda > 0.01 and both signs hold
// more than one node, relabels the group Max+1 / Max+2.
//
// All groups that exist when a round sweep starts are independent, and the
// reference hands out new labels in round order, so processing every pending
// group of a "generation" together and assigning labels in round order
// afterwards gives exactly the reference's labelling.  Per generation the
// induced sub-graphs of all groups are built at once, with columns renumbered
// to positions inside the group, so the power iteration reads the group's own
// contiguous vector.  Then, by size:
//   - small groups: one CTA each; CSR and vectors are staged in shared
//     memory for the whole power iteration, and the two reductions per step
//     are block barriers only;
//   - medium groups: one 16-CTA thread-block cluster each, reductions through
//     distributed shared memory and cluster barriers;
//   - large groups: the whole GPU as one cooperative grid, one fat block per
//     SM so the grid barrier stays short.
// Each step needs only two reductions: |y| for y = B v, then |v' -+ v| and
// v'.k for the next step together.  Reductions are FP64 in a fixed order, so
// results are deterministic.
#include "pg_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>

namespace cg = cooperative_groups;

namespace {
constexpr int GROUP_THREADS = 1024; // one-CTA and cluster power iterations
constexpr int COOP_THREADS = 1024;
constexpr int MAX_ITER = 10000;
constexpr double EPSILON = 1e-6;
constexpr double LAMBDA = 0.01;
constexpr size_t SMEM_CAP = 200 * 1024;        // shared-memory budget of the one-CTA path
constexpr long long MEDIUM_EDGES = 1LL << 22;  // at most this many edges: one cluster per group
constexpr int CLUSTER = 16;                    // CTAs per cluster for medium groups

size_t small_bytes(long long n, long long e)
{
    // sR (n+1 ints), sC (e ints), kdeg, sumBG, v, v0 (n doubles each), 16-byte aligned parts
    return ((size_t)(n + 1) * 4 + 15) / 16 * 16 + ((size_t)e * 4 + 15) / 16 * 16 + (size_t)n * 32;
}

// In-group degree of every member (label of neighbour == label of node).
__global__ void k_nm_gdeg(const int32_t* __restrict__ R, const int32_t* __restrict__ C,
                          const int32_t* __restrict__ label, const int32_t* __restrict__ AD, int32_t P,
                          int32_t* __restrict__ kg)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = gw; p < P; p += nw) {
        int i = AD[p], li = label[i];
        int c = 0;
        for (int32_t q = R[i] + lane; q < R[i + 1]; q += 32) c += label[C[q]] == li;
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) kg[p] = c;
    }
}

// Induced CSR rows in CSR order, columns renumbered to the position of the
// neighbour inside its group (the reference keeps original ids and a
// node-indexed scatter array, which is the same arithmetic).  Group g's n+1
// row offsets (relative to its first edge) sit at sR[goff[g] + g ...].
__global__ void k_nm_gfill(const int32_t* __restrict__ R, const int32_t* __restrict__ C,
                           const int32_t* __restrict__ label, const int32_t* __restrict__ pos,
                           const int32_t* __restrict__ AD, int32_t P, const long long* __restrict__ soff,
                           const long long* __restrict__ goff, const long long* __restrict__ eoff,
                           const int32_t* __restrict__ gidx, int32_t* __restrict__ sR, int32_t* __restrict__ sC)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = gw; p < P; p += nw) {
        const int i = AD[p], li = label[i], q = gidx[p];
        const long long e0 = eoff[q];
        long long w = soff[p];
        if (lane == 0) {
            sR[p + q] = (int32_t)(w - e0);
            if (p + 1 == goff[q + 1]) sR[p + q + 1] = (int32_t)(soff[p + 1] - e0);
        }
        for (int32_t base = R[i]; base < R[i + 1]; base += 32) {
            int32_t e = base + lane;
            bool in = e < R[i + 1] && label[C[e]] == li;
            unsigned m = __ballot_sync(0xffffffffu, in);
            if (in) sC[w + __popc(m & ((1u << lane) - 1u))] = pos[C[e]];
            w += __popc(m);
        }
    }
}

// sumBG (Sub_Partition, Modularity_CPU.cpp:171-173): kg - k * (double)innerM / 2 / M.
__global__ void k_nm_gsumbg(const int32_t* __restrict__ R, const int32_t* __restrict__ AD,
                            const int32_t* __restrict__ kg, const int32_t* __restrict__ gidx,
                            const long long* __restrict__ innerM, int32_t P, int M, double* __restrict__ sumBG,
                            double* __restrict__ kdeg)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        int i = AD[p];
        int k = R[i + 1] - R[i];
        double t = __dmul_rn((double)k, (double)innerM[gidx[p]]);
        t = __ddiv_rn(t, 2.0);
        t = __ddiv_rn(t, (double)M);
        sumBG[p] = __dsub_rn((double)kg[p], t);
        kdeg[p] = (double)k;
    }
}

// One group: rows are the group's members in ascending node id; sR holds
// n+1 offsets into sC, sC holds positions inside the group.
struct Group {
    const int32_t* AD;
    const int32_t* sR;
    const int32_t* sC;
    const double* kdeg;
    const double* sumBG;
    double* v;      // current vector (the reference's v0 entering a step)
    double* v0;     // previous vector; holds y inside a step
    int ng;
};

// The reference's Lead_Vector (Modularity_CPU.cpp:224-298) with two
// reductions per step; `Red` supplies barrier + sum over the threads that own
// the group.
template <class Red>
__device__ double lead_vector(const Group& g, int M, double beta, int* iters, double* resid, Red& red, int tid,
                              int nthr, int lane, int wid, int nwarp)
{
    double x[3];
    double vk = 0.0;
    for (int p = tid; p < g.ng; p += nthr) {
        double vp = (double)g.AD[p];
        g.v[p] = vp;
        vk += vp * g.kdeg[p];
    }
    x[0] = vk;
    red.sum(x, 1);
    vk = x[0];
    double err1 = 1.0, err2 = 1.0, vnorm = 0.0;
    int iter = 0;
    while (err1 > EPSILON && err2 > EPSILON && iter < MAX_ITER) {
        const double c = vk / 2.0 / (double)M;
        double y2 = 0.0;
        for (int p = wid; p < g.ng; p += nwarp) {
            double s = 0.0;
            for (int32_t q = g.sR[p] + lane; q < g.sR[p + 1]; q += 32) s += g.v[g.sC[q]];
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) {
                s -= c * g.kdeg[p] + (g.sumBG[p] - beta) * g.v[p];
                g.v0[p] = s;
                y2 += s * s;
            }
        }
        x[0] = y2;
        red.sum(x, 1);
        vnorm = sqrt(x[0]);
        double e1 = 0.0, e2 = 0.0;
        vk = 0.0;
        for (int p = tid; p < g.ng; p += nthr) {
            const double vold = g.v[p];
            const double vp = g.v0[p] / vnorm;
            const double d1 = vp - vold, d2 = vp + vold;
            e1 += d1 * d1;
            e2 += d2 * d2;
            vk += vp * g.kdeg[p];
            g.v0[p] = vold;
            g.v[p] = vp;
        }
        x[0] = e1;
        x[1] = e2;
        x[2] = vk;
        red.sum(x, 3);
        err1 = sqrt(x[0]);
        err2 = sqrt(x[1]);
        vk = x[2];
        iter++;
    }
    *iters = iter;
    *resid = fmin(err1, err2);
    // first entry of largest magnitude decides the sign (Modularity_CPU.cpp:291-296)
    const int mx = red.argmax_abs(g.v, g.ng, tid, nthr);
    double lam = 0.0;
    if (g.ng > 0) lam = (g.v[mx] * g.v0[mx] > 0) ? vnorm : -vnorm;
    red.sync();
    return lam;
}

struct WarpSlots {
    double warp[32][4];
    double bcast[4];
    int par;
};

__device__ __forceinline__ void warp_reduce(double* x, int k)
{
    for (int q = 0; q < k; q++)
        for (int o = 16; o; o >>= 1) x[q] += __shfl_xor_sync(0xffffffffu, x[q], o);
}

// per-warp (|v|max, first index) over a strided range
__device__ __forceinline__ void local_argmax(const double* v, int n, int tid, int nthr, double& best, int& bi)
{
    best = -1.0;
    bi = 0x7fffffff;
    for (int p = tid; p < n; p += nthr) {
        double m = fabs(v[p]);
        if (m > best) { best = m; bi = p; }
    }
    for (int o = 16; o; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
}

// block-level (value, index) of the warp results, in warp order (thread 0)
__device__ __forceinline__ void block_argmax(const WarpSlots& s, int nw, double& b, int& ix)
{
    b = -1.0;
    ix = 0x7fffffff;
    for (int ww = 0; ww < nw; ww++)
        if (s.warp[ww][0] > b || (s.warp[ww][0] == b && (int)s.warp[ww][1] < ix)) {
            b = s.warp[ww][0];
            ix = (int)s.warp[ww][1];
        }
}

// ---- one CTA owns the group: block barriers only
struct BlockRed {
    WarpSlots s;
    __device__ void sync() { __syncthreads(); }
    __device__ void sum(double* x, int k)
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        warp_reduce(x, k);
        if (lane == 0)
            for (int q = 0; q < k; q++) s.warp[w][q] = x[q];
        __syncthreads();
        if (threadIdx.x < k) {
            double t = 0.0;
            for (int ww = 0; ww < nw; ww++) t += s.warp[ww][threadIdx.x];
            s.bcast[threadIdx.x] = t;
        }
        __syncthreads();
        for (int q = 0; q < k; q++) x[q] = s.bcast[q];
        __syncthreads();
    }
    __device__ int argmax_abs(const double* v, int n, int tid, int nthr)
    {
        double best;
        int bi;
        local_argmax(v, n, tid, nthr, best, bi);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) { s.warp[w][0] = best; s.warp[w][1] = (double)bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double b;
            int ix;
            block_argmax(s, nw, b, ix);
            s.bcast[0] = (double)(ix == 0x7fffffff ? 0 : ix);
        }
        __syncthreads();
        const int r = (int)s.bcast[0];
        __syncthreads();
        return r;
    }
};

// ---- a thread-block cluster owns the group: DSMEM partials, cluster barrier
struct ClusterRed {
    WarpSlots s;
    double slot[2][4];
    __device__ void init()
    {
        if (threadIdx.x == 0) s.par = 0;
        __syncthreads();
    }
    // cluster barriers release/acquire at cluster scope, which orders the
    // global-memory vector writes of one CTA before the reads of another
    __device__ void sync() { cg::this_cluster().sync(); }
    __device__ void sum(double* x, int k)
    {
        cg::cluster_group cl = cg::this_cluster();
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        warp_reduce(x, k);
        if (lane == 0)
            for (int q = 0; q < k; q++) s.warp[w][q] = x[q];
        __syncthreads();
        const int pr = s.par;
        if (threadIdx.x < k) {
            double t = 0.0;
            for (int ww = 0; ww < nw; ww++) t += s.warp[ww][threadIdx.x];
            slot[pr][threadIdx.x] = t;
        }
        // the other slot half is written next; this one again only after
        // another cluster barrier, when every CTA has read it
        cl.sync();
        if (threadIdx.x < k) {
            double t = 0.0;
            for (int r = 0; r < (int)cl.num_blocks(); r++) t += cl.map_shared_rank(this, r)->slot[pr][threadIdx.x];
            s.bcast[threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x == 0) s.par = pr ^ 1;
        for (int q = 0; q < k; q++) x[q] = s.bcast[q];
        __syncthreads();
    }
    __device__ int argmax_abs(const double* v, int n, int tid, int nthr)
    {
        cg::cluster_group cl = cg::this_cluster();
        double best;
        int bi;
        local_argmax(v, n, tid, nthr, best, bi);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) { s.warp[w][0] = best; s.warp[w][1] = (double)bi; }
        __syncthreads();
        const int pr = s.par;
        if (threadIdx.x == 0) {
            double b;
            int ix;
            block_argmax(s, nw, b, ix);
            slot[pr][0] = b;
            slot[pr][1] = (double)ix;
        }
        cl.sync();
        if (threadIdx.x == 0) {
            double b = -1.0;
            int ix = 0x7fffffff;
            for (int r = 0; r < (int)cl.num_blocks(); r++) {
                const ClusterRed* o = cl.map_shared_rank(this, r);
                double ob = o->slot[pr][0];
                int oi = (int)o->slot[pr][1];
                if (ob > b || (ob == b && oi < ix)) { b = ob; ix = oi; }
            }
            s.bcast[0] = (double)(ix == 0x7fffffff ? 0 : ix);
            s.par = pr ^ 1;
        }
        __syncthreads();
        const int r = (int)s.bcast[0];
        __syncthreads();
        return r;
    }
};

// ---- the whole cooperative grid owns the group
struct GridRed {
    WarpSlots s;
    double* part;   // [2][gridDim.x][4], alternate halves per reduction
    __device__ void init(double* p)
    {
        if (threadIdx.x == 0) { part = p; s.par = 0; }
        __syncthreads();
    }
    __device__ void sync() { cg::this_grid().sync(); }
    __device__ void sum(double* x, int k)
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        warp_reduce(x, k);
        if (lane == 0)
            for (int q = 0; q < k; q++) s.warp[w][q] = x[q];
        __syncthreads();
        const int pr = s.par;
        double* pp = part + (size_t)pr * gridDim.x * 4;
        if (threadIdx.x < k) {
            double t = 0.0;
            for (int ww = 0; ww < nw; ww++) t += s.warp[ww][threadIdx.x];
            pp[blockIdx.x * 4 + threadIdx.x] = t;
        }
        // one grid barrier per reduction: the other half of `part` is written
        // next, and this half again only after another barrier
        cg::this_grid().sync();
        if (threadIdx.x < k) {
            double t = 0.0;
            for (int b = 0; b < (int)gridDim.x; b++) t += pp[b * 4 + threadIdx.x];
            s.bcast[threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x == 0) s.par = pr ^ 1;
        for (int q = 0; q < k; q++) x[q] = s.bcast[q];
        __syncthreads();
    }
    __device__ int argmax_abs(const double* v, int n, int tid, int nthr)
    {
        double best;
        int bi;
        local_argmax(v, n, tid, nthr, best, bi);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) { s.warp[w][0] = best; s.warp[w][1] = (double)bi; }
        __syncthreads();
        const int pr = s.par;
        double* pp = part + (size_t)pr * gridDim.x * 4;
        if (threadIdx.x == 0) {
            double b;
            int ix;
            block_argmax(s, nw, b, ix);
            pp[blockIdx.x * 4 + 0] = b;
            pp[blockIdx.x * 4 + 1] = (double)ix;
        }
        cg::this_grid().sync();
        if (threadIdx.x == 0) {
            double b = -1.0;
            int ix = 0x7fffffff;
            for (int r = 0; r < (int)gridDim.x; r++) {
                double ob = pp[r * 4 + 0];
                int oi = (int)pp[r * 4 + 1];
                if (ob > b || (ob == b && oi < ix)) { b = ob; ix = oi; }
            }
            s.bcast[0] = (double)(ix == 0x7fffffff ? 0 : ix);
            s.par = pr ^ 1;
        }
        __syncthreads();
        const int r = (int)s.bcast[0];
        __syncthreads();
        return r;
    }
};

struct Inputs {
    const long long* goff;   // group start in member order (G+1)
    const long long* eoff;   // group start in edge order (G+1)
    const int32_t* AD;
    const int32_t* sR;       // group g's n+1 row offsets start at goff[g] + g
    const int32_t* sC;
    const double* kdeg;
    const double* sumBG;
    double* v;
    double* v0;
    int M;
    int gpu_rule_above;
    double* out;             // per group: lambda, it0, res0, it1, res1, subP, subN, shifted
};

__device__ __forceinline__ Group global_group(const Inputs& in, int gi)
{
    const long long p0 = in.goff[gi];
    Group g;
    g.ng = (int)(in.goff[gi + 1] - p0);
    g.AD = in.AD + p0;
    g.sR = in.sR + p0 + gi;
    g.sC = in.sC + in.eoff[gi];
    g.kdeg = in.kdeg + p0;
    g.sumBG = in.sumBG + p0;
    g.v = in.v + p0;
    g.v0 = in.v0 + p0;
    return g;
}

// Both passes of Sub_Partition for one group.
template <class Red>
__device__ void sub_partition(const Group& g, const Inputs& in, int gi, Red& red, int tid, int nthr, int lane,
                              int wid, int nwarp, bool writer)
{
    int it0, it1 = 0;
    double r0, r1 = 0.0;
    double lam = lead_vector(g, in.M, 0.0, &it0, &r0, red, tid, nthr, lane, wid, nwarp);
    const double below = g.ng > in.gpu_rule_above ? -LAMBDA : 0.0;
    const bool shifted = lam < below;
    if (shifted) lam += lead_vector(g, in.M, -lam, &it1, &r1, red, tid, nthr, lane, wid, nwarp);
    double x[3] = {0.0, 0.0, 0.0};
    for (int p = tid; p < g.ng; p += nthr) {
        x[0] += g.v[p] > 0.0;
        x[1] += g.v[p] <= 0.0;
    }
    red.sum(x, 2);
    if (writer) {
        double* o = in.out + (size_t)gi * 8;
        o[0] = lam; o[1] = it0; o[2] = r0; o[3] = it1; o[4] = r1; o[5] = x[0]; o[6] = x[1]; o[7] = shifted;
    }
}

// small groups: one CTA per group, everything in shared memory
__global__ void __launch_bounds__(GROUP_THREADS)
k_nm_block(const int* __restrict__ glist, Inputs in)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ BlockRed red;
    const int gi = glist[blockIdx.x];
    const Group gg = global_group(in, gi);
    const int n = gg.ng;
    const long long ne = in.eoff[gi + 1] - in.eoff[gi];
    int32_t* sR = (int32_t*)sm;
    int32_t* sC = (int32_t*)(sm + ((size_t)(n + 1) * 4 + 15) / 16 * 16);
    double* dv = (double*)((unsigned char*)sC + ((size_t)ne * 4 + 15) / 16 * 16);
    for (int p = threadIdx.x; p <= n; p += blockDim.x) sR[p] = gg.sR[p];
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
        dv[p] = gg.kdeg[p];
        dv[n + p] = gg.sumBG[p];
    }
    for (long long q = threadIdx.x; q < ne; q += blockDim.x) sC[q] = gg.sC[q];
    __syncthreads();
    Group g = gg;
    g.sR = sR;
    g.sC = sC;
    g.kdeg = dv;
    g.sumBG = dv + n;
    g.v = dv + 2 * n;
    g.v0 = dv + 3 * n;
    sub_partition(g, in, gi, red, threadIdx.x, blockDim.x, threadIdx.x & 31, threadIdx.x >> 5, blockDim.x >> 5,
                  threadIdx.x == 0);
    for (int p = threadIdx.x; p < n; p += blockDim.x) gg.v[p] = g.v[p];   // the labels are assigned from v
}

// medium groups: one cluster per group, global memory
__global__ void __launch_bounds__(GROUP_THREADS)
k_nm_cluster(const int* __restrict__ glist, Inputs in)
{
    __shared__ ClusterRed red;
    cg::cluster_group cl = cg::this_cluster();
    red.init();
    cl.sync();
    const int gi = glist[blockIdx.x / cl.num_blocks()];
    Group g = global_group(in, gi);
    const int ct = (int)cl.block_rank() * blockDim.x + threadIdx.x, cth = (int)cl.num_blocks() * blockDim.x;
    sub_partition(g, in, gi, red, ct, cth, threadIdx.x & 31, ct >> 5, cth >> 5, ct == 0);
    // no CTA may exit while another still reads its shared memory
    cl.sync();
}

// large groups: the whole cooperative grid, one group per launch
__global__ void __launch_bounds__(COOP_THREADS)
k_nm_coop(int gi, Inputs in, double* __restrict__ part)
{
    __shared__ GridRed red;
    red.init(part);
    Group g = global_group(in, gi);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    sub_partition(g, in, gi, red, tid, nthr, threadIdx.x & 31, tid >> 5, nthr >> 5, tid == 0);
}

__global__ void k_nm_gassign(const int32_t* __restrict__ AD, const int32_t* __restrict__ gidx,
                             const double* __restrict__ v, int32_t P, const int* __restrict__ base,
                             const double* __restrict__ coef, int32_t* __restrict__ label)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        int gi = gidx[p];
        if (base[gi] >= 0) label[AD[p]] = base[gi] + 1 + (v[p] * coef[gi] <= 0.0);
    }
}

// Q pieces: edges inside modules and module degree sums (exact integers).
__global__ void k_nm_q(const int32_t* __restrict__ R, const int32_t* __restrict__ C, const int32_t* __restrict__ label,
                       int32_t n, unsigned long long* __restrict__ inside, unsigned long long* __restrict__ Kc)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long in = 0;
    for (int i = gw; i < n; i += nw) {
        int li = label[i];
        unsigned c = 0;
        for (int32_t q = R[i] + lane; q < R[i + 1]; q += 32) c += label[C[q]] == li;
        in += __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) atomicAdd(&Kc[li], (unsigned long long)(R[i + 1] - R[i]));
    }
    if (lane == 0 && in) atomicAdd(inside, in);
}
}  // namespace

extern "C" pg_status pg_newman(pg_ctx* ctx, const pg_graph* g, int32_t gpu_rule_above, int32_t* labels, double* Q,
                               int32_t* n_modules, pg_log_fn log, void* user)
{
    if (!ctx || !g || !labels) return pg_fail(ctx, PG_ERR_INVALID, "pg_newman: null argument");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = g->n;
    const long long nnz = g->nnz;
    const int M = (int)(nnz / 2);
    if (M == 0) {
        // no edges: the reference's power iteration divides by 2M; report one module, Q = 0
        for (int i = 0; i < n; i++) labels[i] = 1;
        if (Q) *Q = 0.0;
        if (n_modules) *n_modules = 1;
        return PG_OK;
    }
    int32_t *label, *AD, *gidx, *kg, *sR, *sC, *dbase, *glist, *pos;
    long long *soff, *goff, *eoff, *innerM;
    double *v, *v0, *sumBG, *kdeg, *part, *out, *dcoef;
    unsigned long long* acc;
    PG_TRY(pg_wst(ctx, "nm.label", (size_t)n + 1, &label));
    PG_TRY(pg_wst(ctx, "nm.AD", (size_t)n + 1, &AD));
    PG_TRY(pg_wst(ctx, "nm.pos", (size_t)n + 1, &pos));
    PG_TRY(pg_wst(ctx, "nm.gidx", (size_t)n + 1, &gidx));
    PG_TRY(pg_wst(ctx, "nm.kg", (size_t)n + 1, &kg));
    PG_TRY(pg_wst(ctx, "nm.soff", (size_t)n + 2, &soff));
    PG_TRY(pg_wst(ctx, "nm.sC", (size_t)nnz + 1, &sC));
    PG_TRY(pg_wst(ctx, "nm.v", (size_t)n + 1, &v));
    PG_TRY(pg_wst(ctx, "nm.v0", (size_t)n + 1, &v0));
    PG_TRY(pg_wst(ctx, "nm.sumBG", (size_t)n + 1, &sumBG));
    PG_TRY(pg_wst(ctx, "nm.kdeg", (size_t)n + 1, &kdeg));
    PG_TRY(pg_wst(ctx, "nm.acc", 4, &acc));
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nm_coop, COOP_THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "power iteration kernel cannot be resident");
    const int coop_grid = ctx->sm_count;   // one fat block per SM keeps the grid barrier short
    PG_TRY(pg_wst(ctx, "nm.part", (size_t)coop_grid * 8 + 8, &part));
    int cluster = CLUSTER;  // 16 needs the non-portable opt-in
    if (cudaFuncSetAttribute(k_nm_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        cluster = 8;
    }
    const size_t smem_cap = std::min(SMEM_CAP, (size_t)ctx->smem_optin - 8192);
    PG_CUDA(ctx, cudaFuncSetAttribute(k_nm_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    PG_CUDA(ctx, cudaMemsetAsync(label, 0, sizeof(int32_t) * (n + 1), ctx->stream));

    std::vector<int32_t> hR(n + 1), hl(n);
    PG_TRY(pg_d2h(ctx, hR.data(), g->R, sizeof(int32_t) * (n + 1)));
    const int grid = ctx->sm_count * 4;
    std::vector<int32_t> adjust((size_t)n + 2, 0);
    int Round = 0, Max_Result = 0, Module_Num = 1, Index = 1;
    char line[512];
    std::vector<int32_t> hAD(n), hgidx(n), hpos(n, 0);
    // wall time per kind of power-iteration launch, reported in the log
    double t_small = 0, t_medium = 0, t_large = 0, t_setup = 0;
    long long it_small = 0, it_medium = 0, it_large = 0;
    int generations = 0;
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto ms_since = [&](std::chrono::steady_clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(now() - t0).count();
    };
    while (Round <= Max_Result) {
        generations++;
        auto t_gen = now();
        // ---- pending groups of this generation: labels Round..Max_Result
        const int lo = Round, hi = Max_Result, G = hi - lo + 1;
        PG_TRY(pg_d2h(ctx, hl.data(), label, sizeof(int32_t) * n));
        std::vector<long long> hgoff(G + 1, 0), hinner(G, 0);
        for (int i = 0; i < n; i++)
            if (hl[i] >= lo && hl[i] <= hi) hgoff[hl[i] - lo + 1]++;
        for (int q = 0; q < G; q++) hgoff[q + 1] += hgoff[q];
        const int P = (int)hgoff[G];
        {
            std::vector<long long> cur(hgoff.begin(), hgoff.end() - 1);
            for (int i = 0; i < n; i++)
                if (hl[i] >= lo && hl[i] <= hi) {
                    int q = hl[i] - lo;
                    hAD[cur[q]] = i;
                    hgidx[cur[q]] = q;
                    hpos[i] = (int32_t)(cur[q] - hgoff[q]);
                    cur[q]++;
                    hinner[q] += hR[i + 1] - hR[i];
                }
        }
        if (P == 0) { Round = hi + 1; continue; }
        PG_TRY(pg_wst(ctx, "nm.sR", (size_t)P + G + 2, &sR));   // n+1 offsets per group
        PG_TRY(pg_wst(ctx, "nm.goff", (size_t)G + 1, &goff));
        PG_TRY(pg_wst(ctx, "nm.eoff", (size_t)G + 1, &eoff));
        PG_TRY(pg_wst(ctx, "nm.inner", (size_t)G, &innerM));
        PG_TRY(pg_wst(ctx, "nm.out", (size_t)G * 8, &out));
        PG_TRY(pg_wst(ctx, "nm.glist", (size_t)G, &glist));
        PG_TRY(pg_wst(ctx, "nm.base", (size_t)G, &dbase));
        PG_TRY(pg_wst(ctx, "nm.coef", (size_t)G, &dcoef));
        PG_CUDA(ctx, cudaMemcpyAsync(AD, hAD.data(), sizeof(int32_t) * P, cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(gidx, hgidx.data(), sizeof(int32_t) * P, cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(pos, hpos.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(goff, hgoff.data(), sizeof(long long) * (G + 1), cudaMemcpyHostToDevice,
                                     ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(innerM, hinner.data(), sizeof(long long) * G, cudaMemcpyHostToDevice,
                                     ctx->stream));
        k_nm_gdeg<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, AD, P, kg);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_scan_counts(ctx, kg, (int64_t*)soff, P));
        std::vector<long long> hsoff(P + 1), heoff(G + 1);
        PG_TRY(pg_d2h(ctx, hsoff.data(), soff, sizeof(long long) * (P + 1)));
        for (int q = 0; q <= G; q++) heoff[q] = hsoff[hgoff[q]];
        PG_CUDA(ctx, cudaMemcpyAsync(eoff, heoff.data(), sizeof(long long) * (G + 1), cudaMemcpyHostToDevice,
                                     ctx->stream));
        k_nm_gfill<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, pos, AD, P, soff, goff, eoff, gidx, sR, sC);
        PG_LAUNCHED(ctx);
        k_nm_gsumbg<<<grid, 256, 0, ctx->stream>>>(g->R, AD, kg, gidx, innerM, P, M, sumBG, kdeg);
        PG_LAUNCHED(ctx);
        t_setup += ms_since(t_gen);
        // ---- power iterations, groups by size
        Inputs in;
        in.goff = goff; in.eoff = eoff; in.AD = AD; in.sR = sR; in.sC = sC; in.kdeg = kdeg; in.sumBG = sumBG;
        in.v = v; in.v0 = v0; in.M = M; in.gpu_rule_above = gpu_rule_above; in.out = out;
        std::vector<int> small, medium, large;
        size_t smem_small = 16;
        for (int q = 0; q < G; q++) {
            const long long ng = hgoff[q + 1] - hgoff[q];
            if (ng == 0) continue;
            const long long edges = heoff[q + 1] - heoff[q];
            const size_t b = small_bytes(ng, edges);
            if (b <= smem_cap) {
                small.push_back(q);
                smem_small = std::max(smem_small, b);
            } else if (edges <= MEDIUM_EDGES && cluster > 1) {
                medium.push_back(q);
            } else {
                large.push_back(q);
            }
        }
        std::vector<double> hout((size_t)G * 8, 0.0);
        std::vector<int> lists(small);
        lists.insert(lists.end(), medium.begin(), medium.end());
        if (!lists.empty())
            PG_CUDA(ctx, cudaMemcpyAsync(glist, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice,
                                         ctx->stream));
        auto t0 = now();
        if (!small.empty()) {
            k_nm_block<<<(int)small.size(), GROUP_THREADS, smem_small, ctx->stream>>>(glist, in);
            PG_LAUNCHED(ctx);
            PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        t_small += ms_since(t0);
        t0 = now();
        if (!medium.empty()) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)(medium.size() * cluster));
            cfg.blockDim = dim3(GROUP_THREADS);
            cfg.stream = ctx->stream;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const int* mlist = glist + small.size();
            PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_nm_cluster, mlist, in));
            PG_LAUNCHED(ctx);
            PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        t_medium += ms_since(t0);
        t0 = now();
        for (int q : large) {
            int qq = q;
            void* args[] = {(void*)&qq, (void*)&in, (void*)&part};
            PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_nm_coop, dim3(coop_grid), dim3(COOP_THREADS), args, 0,
                                                     ctx->stream));
            PG_LAUNCHED(ctx);
        }
        PG_TRY(pg_d2h(ctx, hout.data(), out, sizeof(double) * G * 8));
        t_large += ms_since(t0);
        for (int q : small) it_small += (long long)(hout[(size_t)q * 8 + 1] + hout[(size_t)q * 8 + 3]);
        for (int q : medium) it_medium += (long long)(hout[(size_t)q * 8 + 1] + hout[(size_t)q * 8 + 3]);
        for (int q : large) it_large += (long long)(hout[(size_t)q * 8 + 1] + hout[(size_t)q * 8 + 3]);
        // ---- decisions in round order (labels exactly as the sequential reference)
        std::vector<int> hbase(G, -1);
        std::vector<double> hcoef(G, 0.0);
        bool any_split = false;
        for (int q = 0; q < G; q++) {
            const int round = lo + q;
            const long long ng = hgoff[q + 1] - hgoff[q];
            if (ng == 0) continue;
            const double* o = &hout[(size_t)q * 8];
            const long long subP = (long long)o[5], subN = (long long)o[6];
            const bool issub = o[0] > LAMBDA && subP > 1 && subN > 1;
            if (log) {
                int len = snprintf(line, sizeof line, "Round:\t%d\tnumber of nodes:\t%lld\tIterations:\t%d\tresidual:\t%g\t",
                                   round, ng, (int)o[1], o[2]);
                if (o[7] != 0.0)
                    len += snprintf(line + len, sizeof line - len, "Iterations:\t%d\tresidual:\t%g\t", (int)o[3], o[4]);
                snprintf(line + len, sizeof line - len, "Eigen Value: %g\tDivide?: %d", o[0], (int)issub);
                log(line, user);
            }
            if (issub) {
                hbase[q] = Max_Result;
                hcoef[q] = (double)(subP - subN) + 0.5;
                Max_Result += 2;
                any_split = true;
            } else {
                if (round >= (int)adjust.size()) adjust.resize(round + 1, 0);
                adjust[round] = Index++;
            }
            Module_Num += issub;
        }
        if (any_split) {
            PG_CUDA(ctx, cudaMemcpyAsync(dbase, hbase.data(), sizeof(int) * G, cudaMemcpyHostToDevice, ctx->stream));
            PG_CUDA(ctx, cudaMemcpyAsync(dcoef, hcoef.data(), sizeof(double) * G, cudaMemcpyHostToDevice, ctx->stream));
            k_nm_gassign<<<grid, 256, 0, ctx->stream>>>(AD, gidx, v, P, dbase, dcoef, label);
            PG_LAUNCHED(ctx);
        }
        PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // host vectors above are reused
        Round = hi + 1;
    }
    // Q from module degree sums (Modularity_CPU.cpp:116-124 in closed form)
    unsigned long long* Kc;
    PG_TRY(pg_wst(ctx, "nm.Kc", (size_t)Max_Result + 4, &Kc));
    PG_CUDA(ctx, cudaMemsetAsync(Kc, 0, sizeof(unsigned long long) * (Max_Result + 2), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(unsigned long long), ctx->stream));
    k_nm_q<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, n, acc, Kc);
    PG_LAUNCHED(ctx);
    unsigned long long inside = 0;
    std::vector<unsigned long long> K(Max_Result + 1);
    PG_TRY(pg_d2h(ctx, &inside, acc, sizeof inside));
    PG_TRY(pg_d2h(ctx, K.data(), Kc, sizeof(unsigned long long) * (Max_Result + 1)));
    double sq = 0.0;
    for (int c = 0; c <= Max_Result; c++) sq += (double)K[c] * (double)K[c];
    const double q = ((double)inside - sq / 2 / M) / (2.0 * M);
    PG_TRY(pg_d2h(ctx, hl.data(), label, sizeof(int32_t) * n));
    for (int i = 0; i < n; i++) labels[i] = adjust[hl[i]];
    if (Q) *Q = q;
    if (n_modules) *n_modules = Module_Num;
    if (log) {
        snprintf(line, sizeof line, "Number of Modules: %d,\tQ=%.6g", Module_Num, q);
        log(line, user);
        snprintf(line, sizeof line,
                 "Timing (ms): generations %d, setup %.1f, one-CTA groups %.1f (%lld iterations), "
                 "cluster groups %.1f (%lld), cooperative groups %.1f (%lld)",
                 generations, t_setup, t_small, it_small, t_medium, it_medium, t_large, it_large);
        log(line, user);
    }
    return PG_OK;
}
