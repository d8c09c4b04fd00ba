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
#include <cstring>
#include <string>
#include <thread>

namespace cg = cooperative_groups;

namespace {
constexpr int TEAM_THREADS = 512;   // team power iterations
constexpr int COOP_THREADS = 1024;
constexpr int MAX_ITER = 10000;
constexpr double EPSILON = 1e-6;
constexpr double LAMBDA = 0.01;
constexpr size_t SMEM_CAP = 220 * 1024;        // dynamic shared memory of a team CTA
constexpr long long MEDIUM_EDGES = 1LL << 22;  // at most this many edges: one team per group
constexpr int CLUSTER = 16;                    // largest team (CTAs of one cluster)
constexpr long long MIN_CTA_EDGES = 8192;      // a team CTA keeps at least this many edges
constexpr long long ASYNC_CTA_EDGES = 24576;   // dependency-driven phase: edges per team CTA before doubling
constexpr int RESERVE_SMS = 4;                 // dependency-driven phase: SMs kept free of teams
constexpr size_t POOL_STREAMS = 128;           // dependency-driven phase: streams made ahead
// Per group results: lambda, it0, res0, it1, res1, subP, subN, shifted, and
// the device clock (ns) when its team started and ended.
constexpr int OUT_W = 10;

__device__ __forceinline__ double nm_clock()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (double)t;
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
// row offsets (relative to its first edge) sit at sR[2 goff[g] ...]: twice
// the member offset, so that the offsets of groups nested inside one
// another's member ranges (a group and the children of a finished sibling)
// never overlap.
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
        const long long e0 = eoff[q], g0 = goff[q];
        long long w = soff[p];
        if (lane == 0) {
            sR[g0 + p] = (int32_t)(w - e0);
            if (p + 1 == goff[q + 1]) sR[g0 + p + 1] = (int32_t)(soff[p + 1] - e0);
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

// Children of a split (dependency-driven phase): every member of the batch
// gets its group's id as label and its position inside the group.
__global__ void k_nm_gprep(const int32_t* __restrict__ AD, const int32_t* __restrict__ gidx,
                           const long long* __restrict__ goff, int32_t P, int32_t id0, int32_t* __restrict__ label,
                           int32_t* __restrict__ pos)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int q = gidx[p];
        label[AD[p]] = id0 + q;
        pos[AD[p]] = p - (int)goff[q];
    }
}

// Exclusive prefix sum of the P in-group degrees in one CTA; soff[P] = total,
// copied to pinned host memory (hsoff) before the host's flag is raised.
__global__ void __launch_bounds__(1024) k_nm_gscan(const int32_t* __restrict__ kg, int32_t P,
                                                   long long* __restrict__ soff, long long* __restrict__ hsoff,
                                                   int* __restrict__ hready)
{
    __shared__ long long wsum[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long long carry = 0;
    for (int base = 0; base < P; base += blockDim.x) {
        const int p = base + threadIdx.x;
        const long long x = p < P ? kg[p] : 0;
        long long sc = x;
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, sc, o);
            if (lane >= o) sc += y;
        }
        if (lane == 31) wsum[w] = sc;
        __syncthreads();
        if (w == 0) {
            long long t = lane < nw ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < nw) wsum[lane] = t;
        }
        __syncthreads();
        if (p < P) {
            const long long e = carry + (w ? wsum[w - 1] : 0) + sc - x;
            soff[p] = e;
            hsoff[p] = e;
        }
        carry += wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        soff[P] = carry;
        hsoff[P] = carry;
    }
    // the same offsets in pinned host memory, then the host's flag
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence_system();
        *(volatile int*)hready = 1;
    }
}

__global__ void k_nm_iota(int32_t* __restrict__ x, int32_t n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = i;
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
    // weighted tool: the full graph's values by position, taken at the
    // group's row (wmode 1) or edge (wmode 2) index; wmode 0: no weights
    const float* wv;
    long long wn;
    int wmode;
};

// value at position i of the weight array, 0 past its end
__device__ __forceinline__ double wpos(const float* wv, long long wn, long long i)
{
    return i < wn ? (double)wv[i] : 0.0;
}

// one product term of the weighted tool's SpMV (vv[C[j]] * Vf[..]); the
// product is rounded on its own, as in the reference
template <int WM>
__device__ __forceinline__ double wterm(double x, double w)
{
    return WM == 0 ? x : __dmul_rn(x, w);
}

// Rows of y = B v for the rows this warp owns, L lanes per row.  Each lane
// keeps four independent gathers in flight; the L partial sums meet in a
// shuffle tree.  Returns this lane's share of |y|^2.
template <int L, int WM>
__device__ __forceinline__ double spmv_rows(const Group& g, double c, double beta, int lane, int wid, int nwarp)
{
    constexpr int RPW = 32 / L;
    const int sub = lane & (L - 1);
    double y2 = 0.0;
    for (int base = wid * RPW; base < g.ng; base += nwarp * RPW) {
        const int p = base + lane / L;
        const bool act = p < g.ng;
        int q = 0, q1 = 0;
        if (act) {
            q = g.sR[p] + sub;
            q1 = g.sR[p + 1];
        }
        const double wr = WM == 1 ? wpos(g.wv, g.wn, p) : 1.0;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (; q + 3 * L < q1; q += 4 * L) {
            const int c0 = g.sC[q], c1 = g.sC[q + L], c2 = g.sC[q + 2 * L], c3 = g.sC[q + 3 * L];
            s0 += wterm<WM>(g.v[c0], WM == 2 ? wpos(g.wv, g.wn, q) : wr);
            s1 += wterm<WM>(g.v[c1], WM == 2 ? wpos(g.wv, g.wn, q + L) : wr);
            s2 += wterm<WM>(g.v[c2], WM == 2 ? wpos(g.wv, g.wn, q + 2 * L) : wr);
            s3 += wterm<WM>(g.v[c3], WM == 2 ? wpos(g.wv, g.wn, q + 3 * L) : wr);
        }
        for (; q < q1; q += L) s0 += wterm<WM>(g.v[g.sC[q]], WM == 2 ? wpos(g.wv, g.wn, q) : wr);
        double s = (s0 + s1) + (s2 + s3);
        for (int o = L / 2; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (act && sub == 0) {
            s -= c * g.kdeg[p] + (g.sumBG[p] - beta) * g.v[p];
            g.v0[p] = s;
            y2 += s * s;
        }
    }
    return y2;
}

// Lanes per row: about 8-16 edges per lane, widened while rows alone would
// leave threads idle.  Every thread of a group computes the same value.
__device__ __forceinline__ int lanes_per_row(int ng, long long edges, int nthr)
{
    const long long avg = ng > 0 ? edges / ng : 0;
    int L = 1;
    while (L < 32 && (long long)L * 16 <= avg) L <<= 1;
    while (L < 32 && (long long)ng * L < nthr && 2LL * L <= avg) L <<= 1;
    return L;
}

template <int WM>
__device__ __forceinline__ double spmv_w(int L, const Group& g, double c, double beta, int lane, int wid, int nwarp)
{
    switch (L) {
    case 1: return spmv_rows<1, WM>(g, c, beta, lane, wid, nwarp);
    case 2: return spmv_rows<2, WM>(g, c, beta, lane, wid, nwarp);
    case 4: return spmv_rows<4, WM>(g, c, beta, lane, wid, nwarp);
    case 8: return spmv_rows<8, WM>(g, c, beta, lane, wid, nwarp);
    case 16: return spmv_rows<16, WM>(g, c, beta, lane, wid, nwarp);
    default: return spmv_rows<32, WM>(g, c, beta, lane, wid, nwarp);
    }
}

// W: the kernel is built for the weighted tool (the unweighted build keeps
// none of the weighted code and its register budget)
template <bool W>
__device__ __forceinline__ double spmv(int L, const Group& g, double c, double beta, int lane, int wid, int nwarp)
{
    return (!W || g.wmode == 0) ? spmv_w<0>(L, g, c, beta, lane, wid, nwarp)
           : g.wmode == 1 ? spmv_w<1>(L, g, c, beta, lane, wid, nwarp)
                          : spmv_w<2>(L, g, c, beta, lane, wid, nwarp);
}

// The reference's Lead_Vector (Modularity_CPU.cpp:224-298) with two
// reductions per step; `Red` supplies barrier + sum over the threads that own
// the group.  `ph` alternates the reduction buffers.
template <class Red, bool W>
__device__ double lead_vector(const Group& g, int M, double beta, double err_sq, int* iters, double* resid, Red& red,
                              int tid, int nthr, int lane, int wid, int nwarp, int& ph)
{
    double x[3];
    double vk = 0.0;
    for (int p = tid; p < g.ng; p += nthr) {
        double vp = (double)g.AD[p];
        g.v[p] = vp;
        vk += vp * g.kdeg[p];
    }
    x[0] = vk;
    red.sum(x, 1, ph);
    vk = x[0];
    const int L = lanes_per_row(g.ng, g.ng > 0 ? (long long)g.sR[g.ng] - g.sR[0] : 0, nthr);
    // |v' - v|^2 and |v' + v|^2; sqrt(e) > EPSILON exactly when e > err_sq
    double s1 = 1.0, s2 = 1.0, vnorm = 0.0;
    int iter = 0;
    while (s1 > err_sq && s2 > err_sq && iter < MAX_ITER) {
        const double c = vk * 0.5 / (double)M;   // vk / 2 / M, the same double
        x[0] = spmv<W>(L, g, c, beta, lane, wid, nwarp);
        red.sum(x, 1, ph);
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
        red.sum(x, 3, ph);
        s1 = x[0];
        s2 = x[1];
        vk = x[2];
        iter++;
    }
    *iters = iter;
    *resid = fmin(sqrt(s1), sqrt(s2));
    // first entry of largest magnitude decides the sign (Modularity_CPU.cpp:291-296)
    const int mx = red.argmax_abs(g.v, g.ng, tid, nthr, ph);
    double lam = 0.0;
    if (g.ng > 0) lam = (g.v[mx] * g.v0[mx] > 0) ? vnorm : -vnorm;
    red.sync();
    return lam;
}

__device__ __forceinline__ void warp_reduce(double* x, int k)
{
    for (int q = 0; q < k; q++)
        for (int o = 16; o; o >>= 1) x[q] += __shfl_xor_sync(0xffffffffu, x[q], o);
}

// (value, index) maximum over the lanes, lowest index on ties; all lanes end
// with the result
__device__ __forceinline__ void warp_argmax(double& best, int& bi)
{
    for (int o = 16; o; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
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
    warp_argmax(best, bi);
}

// Per-warp partials of up to four sums, two buffers used alternately: a
// buffer is written again only after another barrier that every warp reaches
// once it has read the buffer.
struct Partials {
    double warp[2][32][4];
};

// Sums of K values over one CTA: every warp folds the warp partials itself in
// the same fixed order, so all threads hold bit-identical sums after a single
// block barrier.
template <int K>
__device__ __forceinline__ void block_sum(Partials& s, double (&x)[K], int& ph)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    warp_reduce(x, K);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; q++) s.warp[ph][w][q] = x[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; q++) x[q] = lane < nw ? s.warp[ph][lane][q] : 0.0;
    warp_reduce(x, K);
    ph ^= 1;
}

// ---- the whole cooperative grid owns the group: one value per block in
// global memory, a grid barrier, then warp 0 of every block folds the block
// values in the same order and broadcasts through shared memory.
struct GridRed {
    Partials s;
    double bc[2][4];
    double* part;   // [2][gridDim.x][4]
    __device__ void init(double* p)
    {
        if (threadIdx.x == 0) part = p;
        __syncthreads();
    }
    __device__ void sync() { cg::this_grid().sync(); }
    __device__ void sum(double* x, int k, int& ph)
    {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        warp_reduce(x, k);
        if (lane == 0)
            for (int q = 0; q < k; q++) s.warp[ph][w][q] = x[q];
        __syncthreads();
        double* pp = part + (size_t)ph * gridDim.x * 4;
        if (w == 0) {
            for (int q = 0; q < k; q++) x[q] = lane < nw ? s.warp[ph][lane][q] : 0.0;
            warp_reduce(x, k);
            if (lane < k) pp[blockIdx.x * 4 + lane] = lane == 0 ? x[0] : lane == 1 ? x[1] : x[2];
        }
        // the other half of `part` is written next, and this one again only
        // after another grid barrier
        cg::this_grid().sync();
        if (w == 0) {
            for (int q = 0; q < k; q++) x[q] = 0.0;
            for (int b = lane; b < (int)gridDim.x; b += 32)
                for (int q = 0; q < k; q++) x[q] += pp[b * 4 + q];
            warp_reduce(x, k);
            if (lane < k) bc[ph][lane] = lane == 0 ? x[0] : lane == 1 ? x[1] : x[2];
        }
        __syncthreads();
        for (int q = 0; q < k; q++) x[q] = bc[ph][q];
        ph ^= 1;
    }
    __device__ int argmax_abs(const double* v, int n, int tid, int nthr, int& ph)
    {
        double best;
        int bi;
        local_argmax(v, n, tid, nthr, best, bi);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) { s.warp[ph][w][0] = best; s.warp[ph][w][1] = (double)bi; }
        __syncthreads();
        double* pp = part + (size_t)ph * gridDim.x * 4;
        if (w == 0) {
            best = lane < nw ? s.warp[ph][lane][0] : -1.0;
            bi = lane < nw ? (int)s.warp[ph][lane][1] : 0x7fffffff;
            warp_argmax(best, bi);
            if (lane == 0) { pp[blockIdx.x * 4 + 0] = best; pp[blockIdx.x * 4 + 1] = (double)bi; }
        }
        cg::this_grid().sync();
        if (w == 0) {
            best = -1.0;
            bi = 0x7fffffff;
            for (int b = lane; b < (int)gridDim.x; b += 32) {
                const double ob = pp[b * 4 + 0];
                const int oi = (int)pp[b * 4 + 1];
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            warp_argmax(best, bi);
            if (lane == 0) bc[ph][0] = (double)(bi == 0x7fffffff ? 0 : bi);
        }
        __syncthreads();
        const int r = (int)bc[ph][0];
        ph ^= 1;
        return r;
    }
};

struct Inputs {
    const long long* goff;   // group start in member order (G+1)
    const long long* eoff;   // group start in edge order (G+1)
    const int32_t* AD;
    const int32_t* sR;       // group g's n+1 row offsets start at 2 goff[g]
    const int32_t* sC;
    const double* kdeg;
    const double* sumBG;
    double* v;
    double* v0;
    int M;
    int gpu_rule_above;
    double err_sq;           // largest double whose square root is at most EPSILON
    const float* wv;         // weighted tool: value array taken by position (null: unweighted)
    long long wn;
    double* out;             // per group: lambda, it0, res0, it1, res1, subP, subN, shifted
    // dependency-driven phase (null otherwise): pinned host memory the teams
    // write directly -- results per group, the final vector by member
    // position, and a flag per group raised last
    double* hout;
    double* hv;
    int* hdone;
};

__device__ __forceinline__ Group global_group(const Inputs& in, int gi)
{
    const long long p0 = in.goff[gi];
    Group g;
    g.ng = (int)(in.goff[gi + 1] - p0);
    g.AD = in.AD + p0;
    g.sR = in.sR + 2 * p0;
    g.sC = in.sC + in.eoff[gi];
    g.kdeg = in.kdeg + p0;
    g.sumBG = in.sumBG + p0;
    g.v = in.v + p0;
    g.v0 = in.v0 + p0;
    g.wv = in.wv;
    g.wn = in.wn;
    g.wmode = in.wv ? (g.ng > in.gpu_rule_above ? 2 : 1) : 0;
    return g;
}

// Both passes of Sub_Partition for one group.
template <class Red, bool W>
__device__ void sub_partition(const Group& g, const Inputs& in, int gi, Red& red, int tid, int nthr, int lane,
                              int wid, int nwarp, bool writer)
{
    int it0, it1 = 0, ph = 0;
    double r0, r1 = 0.0;
    double lam = lead_vector<Red, W>(g, in.M, 0.0, in.err_sq, &it0, &r0, red, tid, nthr, lane, wid, nwarp, ph);
    const double below = g.ng > in.gpu_rule_above ? -LAMBDA : 0.0;
    const bool shifted = lam < below;
    if (shifted) lam += lead_vector<Red, W>(g, in.M, -lam, in.err_sq, &it1, &r1, red, tid, nthr, lane, wid, nwarp, ph);
    double x[3] = {0.0, 0.0, 0.0};
    for (int p = tid; p < g.ng; p += nthr) {
        x[0] += g.v[p] > 0.0;
        x[1] += g.v[p] <= 0.0;
    }
    red.sum(x, 2, ph);
    if (writer) {
        double* o = in.out + (size_t)gi * OUT_W;
        o[0] = lam; o[1] = it0; o[2] = r0; o[3] = it1; o[4] = r1; o[5] = x[0]; o[6] = x[1]; o[7] = shifted;
    }
}

// ---------------------------------------------------------------- teams
// A team is one CTA, or a thread-block cluster of up to 16 CTAs, that owns
// one group.  Every CTA keeps the whole vector of the group in shared memory
// (plus a zero sentinel at index n) and computes y = B v for an
// edge-balanced range of own rows.  A cluster CTA publishes its rows of y in
// global memory (two buffers used alternately) and, after one cluster barrier
// per step, reads all of y back; then every CTA normalises the whole vector
// and forms |y|, |v' -+ v| and v'.k itself, over all rows in one fixed order.
// All CTAs of a team therefore hold bit-identical vectors and sums and take
// the same decisions, with no reduction across CTAs.
//
// The own rows are stored as a sorted sliced ELL matrix in shared memory:
// rows sorted by length (longest first), slices of 32 / L rows with L lanes
// per row, and per slice the 16-bit columns interleaved so that one warp-wide
// load reads element j of every lane; short rows are padded with the
// sentinel column.  A gather of the vector then costs the bank-conflict time
// of one warp-wide shared-memory access per 32 edges, which bounds a step; L
// is chosen per CTA from the sorted lengths.  When the slices do not fit, the
// CTA reads its rows' CSR from global memory instead.

struct SoloTeam {       // one CTA: y stays in shared memory
    static constexpr bool kCluster = false;
    __device__ static void barrier() { __syncthreads(); }
};
struct ClusterTeam {    // a cluster: rows of y meet in global memory
    static constexpr bool kCluster = true;
    // release/acquire at cluster scope orders the global y stores of every
    // CTA before the loads of every other CTA
    __device__ static void barrier() { cg::this_cluster().sync(); }
};

constexpr int TEAM_MAX_ROWS = 12288;   // rows of a team group (its vector fits shared memory)
constexpr int TEAM_NPT = 8;            // vector entries per thread kept in registers during a step

// First local row whose edge offset reaches rank * E / nb.
__host__ __device__ inline int team_split(const int32_t* R, int n, int rank, int nb)
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

__host__ __device__ inline int pow2_at_least(int x)
{
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Byte offsets of the shared-memory parts of one team CTA; the slices take
// what is left.
struct TeamLayout {
    size_t rep, kd, oy, oprev, obg, oR, key, soff, cols, need_min;
};

__host__ __device__ inline size_t team_take(size_t& at, size_t bytes)
{
    const size_t o = at;
    at += (bytes + 15) / 16 * 16;
    return o;
}

__host__ __device__ inline TeamLayout team_layout(int n, int nown)
{
    TeamLayout t;
    size_t at = 0;
    t.rep = team_take(at, (size_t)(n + 1) * 8);
    t.kd = team_take(at, (size_t)n * 4);                       // degrees, exact as float
    t.oy = team_take(at, (size_t)nown * 8);
    t.oprev = team_take(at, (size_t)nown * 8);
    t.obg = team_take(at, (size_t)nown * 8);
    t.oR = team_take(at, (size_t)(nown + 1) * 4);
    t.key = team_take(at, (size_t)pow2_at_least(nown) * 4);   // sort keys, then the row order
    t.soff = team_take(at, (size_t)(nown + 1) * 4);            // slice offsets (entries)
    t.cols = at;
    t.need_min = at;
    return t;
}

struct Team {
    double* rep;          // the group's vector, n entries and a zero at n
    const float* kd;      // degree of every row
    double* oy;           // own rows: y (one-CTA teams)
    double* oprev;        // own rows: vector entering the step
    double* obg;          // own rows: sumBG
    int32_t* oR;          // own rows: offsets into the own edge range
    const uint32_t* perm; // sliced rows: own row of each slot (sorted)
    const int32_t* soff;  // slice s: entries [soff[s], soff[s+1]) of cols
    const uint16_t* cols; // sliced columns
    const int32_t* gcols; // own edges in global memory (unsliced CTAs)
    int L;                // lanes per row
    int nslices;          // 0: unsliced
    int n, r0, nown;
    int e0;               // the group's index of the first own edge
    const float* wv;      // weighted tool, as in Group
    long long wn;
    int wmode;
};

// own rows of y = B v from the sliced matrix, written to ydst[own row]
// (WM = 1: every term of a row times the weight at the row's position)
template <int L, int WM>
__device__ __forceinline__ void team_slices(const Team& tm, double* ydst, double c, double beta, int lane, int wid,
                                            int nwarp)
{
    constexpr int RPS = 32 / L;
    const double* __restrict__ rep = tm.rep;
    const int sub = lane & (L - 1);
    for (int s = wid; s < tm.nslices; s += nwarp) {
        const int b = tm.soff[s], it = (tm.soff[s + 1] - b) >> 5;
        const uint16_t* __restrict__ cs = tm.cols + b + lane;
        double w = 1.0;
        if (WM == 1) {
            const int slot = s * RPS + lane / L;
            w = slot < tm.nown ? wpos(tm.wv, tm.wn, tm.r0 + (int)tm.perm[slot]) : 0.0;
        }
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int j = 0;
        for (; j + 3 < it; j += 4) {
            const int c0 = cs[32 * j], c1 = cs[32 * j + 32], c2 = cs[32 * j + 64], c3 = cs[32 * j + 96];
            a0 += wterm<WM>(rep[c0], w);
            a1 += wterm<WM>(rep[c1], w);
            a2 += wterm<WM>(rep[c2], w);
            a3 += wterm<WM>(rep[c3], w);
        }
        for (; j < it; j++) a0 += wterm<WM>(rep[cs[32 * j]], w);
        double y = (a0 + a1) + (a2 + a3);
        for (int o = L / 2; o; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        const int slot = s * RPS + lane / L;
        if (sub == 0 && slot < tm.nown) {
            const int lp = (int)tm.perm[slot], p = tm.r0 + lp;
            ydst[lp] = y - (c * (double)tm.kd[p] + (tm.obg[lp] - beta) * rep[p]);
        }
    }
}

// own rows of y = B v from the CSR in global memory, L lanes per row
// (WM = 1: weight at the row's position; WM = 2: at the edge's position)
template <int L, int WM>
__device__ __forceinline__ void team_rows(const Team& tm, double* ydst, double c, double beta, int lane, int wid,
                                          int nwarp)
{
    constexpr int RPW = 32 / L;
    const double* __restrict__ rep = tm.rep;
    const int32_t* __restrict__ cols = tm.gcols;
    const int sub = lane & (L - 1);
    for (int base = wid * RPW; base < tm.nown; base += nwarp * RPW) {
        const int lp = base + lane / L;
        const bool act = lp < tm.nown;
        int q = 0, q1 = 0;
        if (act) {
            q = tm.oR[lp] + sub;
            q1 = tm.oR[lp + 1];
        }
        const double wr = WM == 1 ? wpos(tm.wv, tm.wn, tm.r0 + lp) : 1.0;
        const long long qe = tm.e0;   // own edge q is the group's edge e0 + q
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (; q + 3 * L < q1; q += 4 * L) {
            const int c0 = cols[q], c1 = cols[q + L], c2 = cols[q + 2 * L], c3 = cols[q + 3 * L];
            s0 += wterm<WM>(rep[c0], WM == 2 ? wpos(tm.wv, tm.wn, qe + q) : wr);
            s1 += wterm<WM>(rep[c1], WM == 2 ? wpos(tm.wv, tm.wn, qe + q + L) : wr);
            s2 += wterm<WM>(rep[c2], WM == 2 ? wpos(tm.wv, tm.wn, qe + q + 2 * L) : wr);
            s3 += wterm<WM>(rep[c3], WM == 2 ? wpos(tm.wv, tm.wn, qe + q + 3 * L) : wr);
        }
        for (; q < q1; q += L) s0 += wterm<WM>(rep[cols[q]], WM == 2 ? wpos(tm.wv, tm.wn, qe + q) : wr);
        double y = (s0 + s1) + (s2 + s3);
        for (int o = L / 2; o; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (act && sub == 0) {
            const int p = tm.r0 + lp;
            ydst[lp] = y - (c * (double)tm.kd[p] + (tm.obg[lp] - beta) * rep[p]);
        }
    }
}

template <int WM>
__device__ __forceinline__ void team_spmv_w(const Team& tm, double* ydst, double c, double beta, int lane, int wid,
                                            int nwarp)
{
    if (WM != 2 && tm.nslices > 0) {   // edge weights need the CSR's edge positions
        switch (tm.L) {
        case 1: team_slices<1, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        case 2: team_slices<2, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        case 4: team_slices<4, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        case 8: team_slices<8, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        case 16: team_slices<16, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        default: team_slices<32, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
        }
    }
    switch (tm.L) {
    case 1: team_rows<1, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    case 2: team_rows<2, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    case 4: team_rows<4, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    case 8: team_rows<8, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    case 16: team_rows<16, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    default: team_rows<32, WM>(tm, ydst, c, beta, lane, wid, nwarp); return;
    }
}

template <bool W>
__device__ __forceinline__ void team_spmv(const Team& tm, double* ydst, double c, double beta, int lane, int wid,
                                          int nwarp)
{
    if (!W || tm.wmode == 0) team_spmv_w<0>(tm, ydst, c, beta, lane, wid, nwarp);
    else if (tm.wmode == 1) team_spmv_w<1>(tm, ydst, c, beta, lane, wid, nwarp);
    else team_spmv_w<2>(tm, ydst, c, beta, lane, wid, nwarp);
}

// first index of the largest |v| over the whole copy, computed by one CTA
__device__ __forceinline__ int block_argmax_abs(Partials& s, const double* v, int n, int& ph)
{
    double best;
    int bi;
    local_argmax(v, n, threadIdx.x, blockDim.x, best, bi);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { s.warp[ph][w][0] = best; s.warp[ph][w][1] = (double)bi; }
    __syncthreads();
    best = lane < nw ? s.warp[ph][lane][0] : -1.0;
    bi = lane < nw ? (int)s.warp[ph][lane][1] : 0x7fffffff;
    warp_argmax(best, bi);
    ph ^= 1;
    return bi == 0x7fffffff ? 0 : bi;
}

// Lead_Vector (Modularity_CPU.cpp:224-298) for a team: the reference's
// per-entry arithmetic, sums in a fixed order over all rows.
template <class Kind, bool W>
__device__ double team_lead_vector(const Team& tm, const Group& gg, int M, double beta, double err_sq, int* iters,
                                   double* resid, Partials& ps, int& ph)
{
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, wid = tid >> 5, nwarp = nthr >> 5;
    const int n = tm.n;
    double x1[1] = {0.0};
    for (int p = tid; p < n; p += nthr) {
        const double vp = (double)gg.AD[p];
        tm.rep[p] = vp;
        x1[0] += vp * (double)tm.kd[p];
    }
    block_sum(ps, x1, ph);
    double vk = x1[0];
    // |v' - v|^2 and |v' + v|^2; sqrt(e) > EPSILON exactly when e > err_sq
    double s1 = 1.0, s2 = 1.0, vnorm = 0.0;
    int iter = 0, yb = 0;
    while (s1 > err_sq && s2 > err_sq && iter < MAX_ITER) {
        const double c = vk * 0.5 / (double)M;   // vk / 2 / M, the same double
        double* ybuf = Kind::kCluster ? (yb ? gg.v0 : gg.v) : tm.oy;
        team_spmv<W>(tm, Kind::kCluster ? ybuf + tm.r0 : ybuf, c, beta, lane, wid, nwarp);
        Kind::barrier();
        double x3[3] = {0.0, 0.0, 0.0};
        if (n <= TEAM_NPT * nthr) {
            // at most TEAM_NPT entries per thread: y is loaded once, all loads
            // and divisions of a thread issued together; the per-thread sums
            // run over p = tid, tid + nthr, ... as in the loops below
            double yv[TEAM_NPT];
            x1[0] = 0.0;
#pragma unroll
            for (int k = 0; k < TEAM_NPT; k++) {
                const int p = tid + k * nthr;
                yv[k] = p < n ? ybuf[p] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < TEAM_NPT; k++)
                if (tid + k * nthr < n) x1[0] += yv[k] * yv[k];
            block_sum(ps, x1, ph);
            vnorm = sqrt(x1[0]);
#pragma unroll
            for (int k = 0; k < TEAM_NPT; k++) {
                const int p = tid + k * nthr;
                if (p < n) {
                    const double vold = tm.rep[p];
                    const double vp = yv[k] / vnorm;
                    const double d1 = vp - vold, d2 = vp + vold;
                    x3[0] += d1 * d1;
                    x3[1] += d2 * d2;
                    x3[2] += vp * (double)tm.kd[p];
                    if ((unsigned)(p - tm.r0) < (unsigned)tm.nown) tm.oprev[p - tm.r0] = vold;
                    tm.rep[p] = vp;
                }
            }
        } else {
            x1[0] = 0.0;
            for (int p = tid; p < n; p += nthr) {
                const double y = ybuf[p];
                x1[0] += y * y;
            }
            block_sum(ps, x1, ph);
            vnorm = sqrt(x1[0]);
            for (int p = tid; p < n; p += nthr) {
                const double vold = tm.rep[p];
                const double vp = ybuf[p] / vnorm;
                const double d1 = vp - vold, d2 = vp + vold;
                x3[0] += d1 * d1;
                x3[1] += d2 * d2;
                x3[2] += vp * (double)tm.kd[p];
                if ((unsigned)(p - tm.r0) < (unsigned)tm.nown) tm.oprev[p - tm.r0] = vold;
                tm.rep[p] = vp;
            }
        }
        block_sum(ps, x3, ph);
        s1 = x3[0];
        s2 = x3[1];
        vk = x3[2];
        yb ^= 1;
        iter++;
    }
    *iters = iter;
    *resid = fmin(sqrt(s1), sqrt(s2));
    // the labels are assigned from v; the sign test below reads v0 of any row
    Kind::barrier();   // the y buffers are free again
    for (int lp = tid; lp < tm.nown; lp += nthr) {
        gg.v[tm.r0 + lp] = tm.rep[tm.r0 + lp];
        gg.v0[tm.r0 + lp] = tm.oprev[lp];
    }
    Kind::barrier();
    // first entry of largest magnitude decides the sign (Modularity_CPU.cpp:291-296)
    const int mx = block_argmax_abs(ps, tm.rep, n, ph);
    const double lam = (tm.rep[mx] * gg.v0[mx] > 0) ? vnorm : -vnorm;
    Kind::barrier();   // every read of the copy and of v0 is done before they change
    return lam;
}

// Sliced layout of the own rows: sort, choose L, fill.  The slices go to
// shared memory (`cols`, `space` bytes) when some L fits there, else to the
// CTA's region of global memory (`gcols`, `gspace` bytes, which always holds
// L = 32).  Returns the number of slices and sets tm.cols.
__device__ int team_slice(Team& tm, const Group& gg, int e0, uint32_t* key, int32_t* soff, uint16_t* cols,
                          size_t space, uint16_t* gcols, size_t gspace, int* sL, int* sIn)
{
    const int tid = threadIdx.x, nthr = blockDim.x, nown = tm.nown;
    const int P2 = pow2_at_least(nown);
    // keys: (65535 - length) << 16 | row, so ascending order is longest
    // first with rows in order on ties
    for (int i = tid; i < P2; i += nthr) {
        uint32_t k = 0xffffffffu;
        if (i < nown) {
            const int len = min(tm.oR[i + 1] - tm.oR[i], 65535);
            k = ((uint32_t)(65535 - len) << 16) | (uint32_t)i;
        }
        key[i] = k;
    }
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < P2; i += nthr) {
                const int o = i ^ j;
                if (o > i) {
                    const uint32_t a = key[i], b = key[o];
                    if ((a > b) == ((i & k) == 0)) {
                        key[i] = b;
                        key[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = tid; i < nown; i += nthr) key[i] &= 0xffffu;   // now the row order
    __syncthreads();
    // cost of lanes-per-row L = 2^t: warp 0 takes the first slice of every
    // round, the longest, so its total bounds the step; a slice costs its
    // gathers plus a fixed 16 (loop, shuffle tree and row store: measured on
    // 16-CTA teams of the 58k graphs, where a smaller constant picked L = 16
    // for some CTAs and made them 20 % slower than their L = 8 neighbours)
    __shared__ long long cost[6], size[6];
    if (tid < 6) {
        const int L = 1 << tid, RPS = 32 / L, ns = (nown + RPS - 1) / RPS, nw = nthr >> 5;
        long long c = 0, sz = 0;
        for (int s = 0; s < ns; s++) {
            const int first = (int)key[s * RPS];
            const int it = (tm.oR[first + 1] - tm.oR[first] + L - 1) / L;
            sz += 32LL * it;
            if (s % nw == 0) c += it + 16 + tid;
        }
        cost[tid] = c;
        size[tid] = sz;
    }
    __syncthreads();
    if (tid == 0) {
        int best = -1;
        for (int t = 0; t < 6; t++)
            if ((size_t)size[t] * 2 <= space && (best < 0 || cost[t] < cost[best])) best = t;
        *sIn = best >= 0;   // in shared memory
        if (best < 0)
            for (int t = 0; t < 6; t++)
                if ((size_t)size[t] * 2 <= gspace && (best < 0 || cost[t] < cost[best])) best = t;
        *sL = best < 0 ? 0 : 1 << best;
        if (best >= 0) {
            const int L = 1 << best, RPS = 32 / L, ns = (nown + RPS - 1) / RPS;
            int at = 0;
            for (int s = 0; s < ns; s++) {
                soff[s] = at;
                const int first = (int)key[s * RPS];
                at += 32 * ((tm.oR[first + 1] - tm.oR[first] + L - 1) / L);
            }
            soff[ns] = at;
        }
    }
    __syncthreads();
    const int L = *sL;
    if (L == 0) return 0;
    if (!*sIn) cols = gcols;
    tm.cols = cols;
    const int RPS = 32 / L, ns = (nown + RPS - 1) / RPS;
    const int lane = tid & 31, sub = lane & (L - 1);
    for (int s = tid >> 5; s < ns; s += nthr >> 5) {
        const int slot = s * RPS + lane / L;
        int q0 = 0, len = 0;
        if (slot < nown) {
            const int r = (int)key[slot];
            q0 = tm.oR[r];
            len = tm.oR[r + 1] - q0;
        }
        const int it = (soff[s + 1] - soff[s]) >> 5;
        for (int j = 0; j < it; j++) {
            const int k = j * L + sub;
            cols[soff[s] + 32 * j + lane] = (uint16_t)(k < len ? gg.sC[e0 + q0 + k] : tm.n);
        }
    }
    __syncthreads();
    return ns;
}

// One team per group of `glist`; the cluster size is set at launch.
template <class Kind, bool W>
__global__ void __launch_bounds__(TEAM_THREADS)
k_nm_team(const int* __restrict__ glist, Inputs in, int smem_bytes, uint16_t* __restrict__ slices)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ Partials ps;
    __shared__ int sL, sIn;
    const double t_start = nm_clock();
    cg::cluster_group cl = cg::this_cluster();
    const int nb = Kind::kCluster ? (int)cl.num_blocks() : 1, rank = Kind::kCluster ? (int)cl.block_rank() : 0;
    const int gi = glist[blockIdx.x / nb];
    const Group gg = global_group(in, gi);
    Team tm;
    tm.n = gg.ng;
    tm.r0 = team_split(gg.sR, tm.n, rank, nb);
    const int r1 = team_split(gg.sR, tm.n, rank + 1, nb);
    tm.nown = r1 - tm.r0;
    const int e0 = gg.sR[tm.r0];
    const TeamLayout t = team_layout(tm.n, tm.nown);
    tm.rep = (double*)(sm + t.rep);
    float* kd = (float*)(sm + t.kd);
    tm.kd = kd;
    tm.oy = (double*)(sm + t.oy);
    tm.oprev = (double*)(sm + t.oprev);
    tm.obg = (double*)(sm + t.obg);
    tm.oR = (int32_t*)(sm + t.oR);
    for (int p = threadIdx.x; p < tm.n; p += blockDim.x) kd[p] = (float)gg.kdeg[p];
    for (int lp = threadIdx.x; lp < tm.nown; lp += blockDim.x) tm.obg[lp] = gg.sumBG[tm.r0 + lp];
    for (int lp = threadIdx.x; lp <= tm.nown; lp += blockDim.x) tm.oR[lp] = gg.sR[tm.r0 + lp] - e0;
    if (threadIdx.x == 0) tm.rep[tm.n] = 0.0;   // the padding column
    __syncthreads();
    uint32_t* key = (uint32_t*)(sm + t.key);
    int32_t* soff = (int32_t*)(sm + t.soff);
    uint16_t* cols = (uint16_t*)(sm + t.cols);
    const size_t space = (size_t)smem_bytes > t.cols ? (size_t)smem_bytes - t.cols : 0;
    // this CTA's region of the global slice store: 2 entries per edge and 64
    // per row, counted from the group's first edge and row
    const long long own_e = (long long)tm.oR[tm.nown];
    uint16_t* gcols = slices + 2 * (in.eoff[gi] + e0) + 64 * (in.goff[gi] + tm.r0);
    const size_t gspace = (size_t)(2 * own_e + 64LL * tm.nown) * 2;
    tm.e0 = e0;
    tm.wv = gg.wv;
    tm.wn = gg.wn;
    tm.wmode = gg.wmode;
    tm.nslices = (tm.n < 65535 && gg.wmode != 2) ? team_slice(tm, gg, e0, key, soff, cols, space, gcols, gspace, &sL, &sIn)
                                                  : 0;
    tm.perm = key;
    tm.soff = soff;
    tm.gcols = gg.sC + e0;
    tm.L = tm.nslices > 0 ? sL : lanes_per_row(tm.nown, tm.nown > 0 ? (long long)tm.oR[tm.nown] : 0, blockDim.x);
    // both passes of Sub_Partition
    int it0, it1 = 0, ph = 0;
    double res0, res1 = 0.0;
    double lam = team_lead_vector<Kind, W>(tm, gg, in.M, 0.0, in.err_sq, &it0, &res0, ps, ph);
    const double below = gg.ng > in.gpu_rule_above ? -LAMBDA : 0.0;
    const bool shifted = lam < below;
    if (shifted) lam += team_lead_vector<Kind, W>(tm, gg, in.M, -lam, in.err_sq, &it1, &res1, ps, ph);
    double x2[2] = {0.0, 0.0};
    for (int p = threadIdx.x; p < tm.n; p += blockDim.x) {
        x2[0] += tm.rep[p] > 0.0;
        x2[1] += tm.rep[p] <= 0.0;
    }
    block_sum(ps, x2, ph);
    double o[OUT_W] = {lam, (double)it0, res0, (double)it1, res1, x2[0], x2[1], (double)shifted, t_start, 0.0};
    if (rank == 0 && threadIdx.x == 0) {
        o[9] = nm_clock();
        for (int k = 0; k < OUT_W; k++) in.out[(size_t)gi * OUT_W + k] = o[k];
    }
    if (in.hdone) {
        // straight to the host: every CTA its own rows of the vector, then
        // (after every CTA's system-scope fence and a team barrier) the
        // results and the flag, so the host sees all of it once the flag is up
        const long long p0 = in.goff[gi];
        for (int lp = threadIdx.x; lp < tm.nown; lp += blockDim.x) in.hv[p0 + tm.r0 + lp] = tm.rep[tm.r0 + lp];
        __threadfence_system();
        Kind::barrier();
        if (rank == 0 && threadIdx.x == 0) {
            for (int k = 0; k < OUT_W; k++) in.hout[(size_t)gi * OUT_W + k] = o[k];
            __threadfence_system();
            *(volatile int*)(in.hdone + gi) = 1;
        }
    }
}

// large groups: the whole cooperative grid, one group per launch
template <bool W>
__global__ void __launch_bounds__(COOP_THREADS)
k_nm_coop(int gi, Inputs in, double* __restrict__ part)
{
    __shared__ GridRed red;
    red.init(part);
    Group g = global_group(in, gi);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    sub_partition<GridRed, W>(g, in, gi, red, tid, nthr, threadIdx.x & 31, tid >> 5, nthr >> 5, tid == 0);
}

// ---------------------------------------------------------------- whole grid
// Groups too large for a team run on the whole GPU as one cooperative grid,
// one group per launch.  Each CTA owns an edge-balanced range of rows; the
// vector lives in global memory.  A step walks the vector in column blocks
// of 2^cb_log entries: every CTA copies a block into shared memory and adds
// the block's share of each own row.  The columns of a row are sorted, so a
// row's edges split into one contiguous range per block, found once per
// launch by binary search; columns are read as 16-bit offsets inside their
// block (a copy made once per launch), which halves the column traffic of a
// step and keeps it in L2.  Two grid-wide reductions per step as in
// Lead_Vector.

struct GridLayout {
    size_t vblk, vown, prev, kdo, bgo, ypart, split, need;
};

__host__ __device__ inline GridLayout grid_layout(int nown, int nblk, int cb)
{
    GridLayout t;
    size_t at = 0;
    t.vblk = team_take(at, (size_t)cb * 8);
    t.vown = team_take(at, (size_t)nown * 8);
    t.prev = team_take(at, (size_t)nown * 8);
    t.kdo = team_take(at, (size_t)nown * 8);
    t.bgo = team_take(at, (size_t)nown * 8);
    t.ypart = team_take(at, (size_t)nown * 8);
    t.split = team_take(at, (size_t)(nblk + 1) * nown * 4);
    t.need = at;
    return t;
}

struct GridPart {
    double *vblk, *vown, *prev, *kdo, *bgo, *ypart;
    const int32_t* split;    // [own row][nblk + 1] edge offsets (global edge index in the group)
    const uint16_t* c16;     // the group's columns modulo the block size
    int n, r0, nown, nblk, cb_log;
    const float* wv;         // weighted tool, as in Group
    long long wn;
    int wmode;
};

// add block b's share of every own row to ypart, L lanes per row
template <int L, int WM>
__device__ __forceinline__ void grid_rows(const GridPart& gp, int b, int lane, int wid, int nwarp)
{
    constexpr int RPW = 32 / L;
    const int sub = lane & (L - 1);
    const double* __restrict__ vb = gp.vblk;
    const uint16_t* __restrict__ cols = gp.c16;
    for (int base = wid * RPW; base < gp.nown; base += nwarp * RPW) {
        const int lp = base + lane / L;
        const bool act = lp < gp.nown;
        int q = 0, q1 = 0;
        if (act) {
            q = gp.split[lp * (gp.nblk + 1) + b] + sub;
            q1 = gp.split[lp * (gp.nblk + 1) + b + 1];
        }
        const double wr = WM == 1 ? wpos(gp.wv, gp.wn, gp.r0 + lp) : 1.0;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (; q + 3 * L < q1; q += 4 * L) {
            const int c0 = cols[q], c1 = cols[q + L], c2 = cols[q + 2 * L], c3 = cols[q + 3 * L];
            s0 += wterm<WM>(vb[c0], WM == 2 ? wpos(gp.wv, gp.wn, q) : wr);
            s1 += wterm<WM>(vb[c1], WM == 2 ? wpos(gp.wv, gp.wn, q + L) : wr);
            s2 += wterm<WM>(vb[c2], WM == 2 ? wpos(gp.wv, gp.wn, q + 2 * L) : wr);
            s3 += wterm<WM>(vb[c3], WM == 2 ? wpos(gp.wv, gp.wn, q + 3 * L) : wr);
        }
        for (; q < q1; q += L) s0 += wterm<WM>(vb[cols[q]], WM == 2 ? wpos(gp.wv, gp.wn, q) : wr);
        double y = (s0 + s1) + (s2 + s3);
        for (int o = L / 2; o; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (act && sub == 0) gp.ypart[lp] = b == 0 ? y : gp.ypart[lp] + y;
    }
}

template <int WM>
__device__ __forceinline__ void grid_block_w(int L, const GridPart& gp, int b, int lane, int wid, int nwarp)
{
    switch (L) {
    case 1: grid_rows<1, WM>(gp, b, lane, wid, nwarp); return;
    case 2: grid_rows<2, WM>(gp, b, lane, wid, nwarp); return;
    case 4: grid_rows<4, WM>(gp, b, lane, wid, nwarp); return;
    case 8: grid_rows<8, WM>(gp, b, lane, wid, nwarp); return;
    case 16: grid_rows<16, WM>(gp, b, lane, wid, nwarp); return;
    default: grid_rows<32, WM>(gp, b, lane, wid, nwarp); return;
    }
}

template <bool W>
__device__ __forceinline__ void grid_block(int L, const GridPart& gp, int b, int lane, int wid, int nwarp)
{
    if (!W || gp.wmode == 0) grid_block_w<0>(L, gp, b, lane, wid, nwarp);
    else if (gp.wmode == 1) grid_block_w<1>(L, gp, b, lane, wid, nwarp);
    else grid_block_w<2>(L, gp, b, lane, wid, nwarp);
}

// Lead_Vector (Modularity_CPU.cpp:224-298) on the whole grid
template <bool W>
__device__ double grid_lead_vector(const GridPart& gp, const Group& gg, int M, double beta, double err_sq, int* iters,
                                   double* resid, GridRed& red, int& ph)
{
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, wid = tid >> 5, nwarp = nthr >> 5;
    double x[3];
    double vk = 0.0;
    for (int lp = tid; lp < gp.nown; lp += nthr) {
        const double vp = (double)gg.AD[gp.r0 + lp];
        gp.vown[lp] = vp;
        gg.v[gp.r0 + lp] = vp;
        vk += vp * gp.kdo[lp];
    }
    x[0] = vk;
    red.sum(x, 1, ph);   // also publishes the start vector
    vk = x[0];
    const long long own_edges = gp.nown > 0 ? (long long)gp.split[gp.nown * (gp.nblk + 1) - 1] - gp.split[0] : 0;
    const int L = lanes_per_row(gp.nown, own_edges / gp.nblk, nthr);
    const int cb = 1 << gp.cb_log;
    double s1 = 1.0, s2 = 1.0, vnorm = 0.0;
    int iter = 0;
    while (s1 > err_sq && s2 > err_sq && iter < MAX_ITER) {
        const double c = vk * 0.5 / (double)M;   // vk / 2 / M, the same double
        for (int b = 0; b < gp.nblk; b++) {
            const int len = min(cb, gp.n - b * cb);
            const double* src = gg.v + (size_t)b * cb;
            for (int p = tid; p < len; p += nthr) gp.vblk[p] = src[p];
            __syncthreads();
            grid_block<W>(L, gp, b, lane, wid, nwarp);
            __syncthreads();
        }
        double y2 = 0.0;
        for (int lp = tid; lp < gp.nown; lp += nthr) {
            const double y = gp.ypart[lp] - (c * gp.kdo[lp] + (gp.bgo[lp] - beta) * gp.vown[lp]);
            gp.ypart[lp] = y;
            y2 += y * y;
        }
        x[0] = y2;
        red.sum(x, 1, ph);
        vnorm = sqrt(x[0]);
        double e1 = 0.0, e2 = 0.0;
        vk = 0.0;
        for (int lp = tid; lp < gp.nown; lp += nthr) {
            const double vold = gp.vown[lp];
            const double vp = gp.ypart[lp] / vnorm;
            const double d1 = vp - vold, d2 = vp + vold;
            e1 += d1 * d1;
            e2 += d2 * d2;
            vk += vp * gp.kdo[lp];
            gp.prev[lp] = vold;
            gp.vown[lp] = vp;
            gg.v[gp.r0 + lp] = vp;
        }
        x[0] = e1;
        x[1] = e2;
        x[2] = vk;
        red.sum(x, 3, ph);   // also publishes the new vector
        s1 = x[0];
        s2 = x[1];
        vk = x[2];
        iter++;
    }
    *iters = iter;
    *resid = fmin(sqrt(s1), sqrt(s2));
    for (int lp = tid; lp < gp.nown; lp += nthr) gg.v0[gp.r0 + lp] = gp.prev[lp];
    red.sync();
    // first entry of largest magnitude decides the sign (Modularity_CPU.cpp:291-296)
    const int gt = blockIdx.x * blockDim.x + tid, gn = gridDim.x * blockDim.x;
    const int mx = red.argmax_abs(gg.v, gp.n, gt, gn, ph);
    const double lam = (gg.v[mx] * gg.v0[mx] > 0) ? vnorm : -vnorm;
    red.sync();   // every read of v and v0 is done before they change
    return lam;
}

template <bool W>
__global__ void __launch_bounds__(COOP_THREADS)
k_nm_grid(int gi, Inputs in, double* __restrict__ part, uint16_t* __restrict__ c16, int cb_log)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ GridRed red;
    red.init(part);
    const Group gg = global_group(in, gi);
    GridPart gp;
    gp.n = gg.ng;
    gp.cb_log = cb_log;
    gp.wv = gg.wv;
    gp.wn = gg.wn;
    gp.wmode = gg.wmode;
    const int cb = 1 << cb_log;
    gp.nblk = (gp.n + cb - 1) >> cb_log;
    gp.r0 = team_split(gg.sR, gp.n, blockIdx.x, gridDim.x);
    const int r1 = team_split(gg.sR, gp.n, blockIdx.x + 1, gridDim.x);
    gp.nown = r1 - gp.r0;
    const GridLayout t = grid_layout(gp.nown, gp.nblk, cb);
    gp.vblk = (double*)(sm + t.vblk);
    gp.vown = (double*)(sm + t.vown);
    gp.prev = (double*)(sm + t.prev);
    gp.kdo = (double*)(sm + t.kdo);
    gp.bgo = (double*)(sm + t.bgo);
    gp.ypart = (double*)(sm + t.ypart);
    int32_t* split = (int32_t*)(sm + t.split);
    gp.split = split;
    uint16_t* cg16 = c16 + in.eoff[gi];
    gp.c16 = cg16;
    // own edges: 16-bit offsets inside their column block
    for (int q = gg.sR[gp.r0] + threadIdx.x; q < gg.sR[r1]; q += blockDim.x)
        cg16[q] = (uint16_t)(gg.sC[q] & (cb - 1));
    for (int lp = threadIdx.x; lp < gp.nown; lp += blockDim.x) {
        const int p = gp.r0 + lp;
        gp.kdo[lp] = gg.kdeg[p];
        gp.bgo[lp] = gg.sumBG[p];
        const int a = gg.sR[p], e = gg.sR[p + 1];
        int32_t* sp = split + lp * (gp.nblk + 1);
        sp[0] = a;
        for (int b = 1; b < gp.nblk; b++) {
            int lo = a, hi = e;   // first edge whose column is at least b * cb
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (gg.sC[mid] >= b * cb) hi = mid;
                else lo = mid + 1;
            }
            sp[b] = lo;
        }
        sp[gp.nblk] = e;
    }
    __syncthreads();
    int it0, it1 = 0, ph = 0;
    double res0, res1 = 0.0;
    double lam = grid_lead_vector<W>(gp, gg, in.M, 0.0, in.err_sq, &it0, &res0, red, ph);
    const double below = gg.ng > in.gpu_rule_above ? -LAMBDA : 0.0;
    const bool shifted = lam < below;
    if (shifted) lam += grid_lead_vector<W>(gp, gg, in.M, -lam, in.err_sq, &it1, &res1, red, ph);
    double x[3] = {0.0, 0.0, 0.0};
    for (int lp = threadIdx.x; lp < gp.nown; lp += blockDim.x) {
        x[0] += gp.vown[lp] > 0.0;
        x[1] += gp.vown[lp] <= 0.0;
    }
    red.sum(x, 2, ph);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* o = in.out + (size_t)gi * OUT_W;
        o[0] = lam; o[1] = it0; o[2] = res0; o[3] = it1; o[4] = res1; o[5] = x[0]; o[6] = x[1]; o[7] = shifted;
    }
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

// ------------------------------------------------------- dependency-driven phase
// Once every pending group fits a team, groups stop waiting for the rest of
// their generation.  Each group's power iteration is a launch of its own on
// a stream of its own, and the team writes its results and final vector
// straight into pinned host memory and then raises a flag there; the host
// polls the flags, decides a group at once and, on a split, builds the two
// children's sub-graphs and launches them.  (Host functions queued behind
// the teams were tried first: a host function holds the hardware queue it
// shares with other streams until the team before it ends, which delayed
// unrelated launches by tens of ms.)  Labels are handed out afterwards by
// replaying the reference's round order over the finished tree, so they are
// those of the sequential reference.
//
// Buffers nest: a group owns member positions [s, s + n) and induced edges
// [es, es + E); its children's positions and edges are subranges of those
// (a child's induced edges are edges of its parent's sub-graph).  Arrays
// with one entry per member (AD, gidx, kg, v, v0, kdeg, sumBG) are indexed
// by position, the scan and sR of a batch (its n + 1 or n + 2 entries) at
// twice the batch's first position; groups in flight own disjoint ranges,
// so none of these overlap.  The member and edge offsets of a batch's two
// groups are read by each team when it starts, which may be after its
// sibling has ended and split at the same first position, so they sit in
// slots of their own, four per batch.
using TeamFn = void (*)(const int*, Inputs, int, uint16_t*);

struct NmAsync {
    struct Node {
        int s = 0, n = 0;
        long long es = 0, E = 0;
        int c = 1;
        int stream = -1;
        int child = -1;        // tree index of the first child; the second follows
        bool split = false;
        bool grid = false;     // ran on the whole grid before the phase began
        int parent = -1;
        double out[OUT_W] = {};
        // launch arguments, kept while the group waits for SMs
        Inputs in = {};
        int gi = 0;
        uint16_t* sl = nullptr;
        cudaEvent_t dep = nullptr;   // the stream waits for this event first
    };
    struct Batch {
        int s, P, nA, first, stream;
        long long es;
    };
    pg_ctx* ctx;
    const pg_graph* g;
    TeamFn k_solo, k_clu;
    Inputs base;               // M, err_sq, gpu_rule_above, weights
    int lo;                    // device label of tree index 0
    size_t smem_cap;
    int max_cluster;
    long long cta_edges;       // a team doubles its CTAs while each holds more edges than this
    const int32_t* hR;
    int32_t *label, *pos, *AD, *gidx, *kg, *sR, *sC, *iota;
    long long *agoff, *aeoff, *asoff, *ainner;
    double *v, *v0, *sumBG, *kdeg, *aout;
    uint16_t* slices;
    int32_t *hAD, *hgidx;
    long long *hsoff, *hgoff, *heoff, *hinner;
    double *hv, *hout;
    std::vector<Node> tree;
    std::vector<Batch> batches;
    // pinned host flags raised by the device: a team's end (per tree node)
    // and a batch's scan (per batch)
    int *hdone, *hready;
    // the same pinned buffers as the device addresses them
    double *dhout, *dhv;
    long long* dhsoff;
    int *dhdone, *dhready;

    pg_status map_pinned()
    {
        PG_CUDA(ctx, cudaHostGetDevicePointer((void**)&dhout, hout, 0));
        PG_CUDA(ctx, cudaHostGetDevicePointer((void**)&dhv, hv, 0));
        PG_CUDA(ctx, cudaHostGetDevicePointer((void**)&dhsoff, hsoff, 0));
        PG_CUDA(ctx, cudaHostGetDevicePointer((void**)&dhdone, hdone, 0));
        PG_CUDA(ctx, cudaHostGetDevicePointer((void**)&dhready, hready, 0));
        return PG_OK;
    }
    std::vector<int> free_streams, running, waiting, queued;
    std::vector<cudaEvent_t> events;
    // team CTAs in flight and their cap: a team CTA holds a whole SM
    // (registers and shared memory), so SMs beyond the cap stay free for the
    // small kernels that build the next children; without it those kernels
    // queued behind the teams for tens of ms
    int inflight = 0, budget = 0;
    bool no_fit = false;       // a child too large for a team (only after an early start)

    pg_status take_stream(int* out)
    {
        if (!free_streams.empty()) {
            *out = free_streams.back();
            free_streams.pop_back();
            return PG_OK;
        }
        PG_TRY(pg_stream_pool(ctx, ctx->pool.size() + 1));
        *out = (int)ctx->pool.size() - 1;
        return PG_OK;
    }

    // CTAs of a group's team: the fewest whose shared memory holds the
    // group, doubled while each CTA keeps more than cta_edges edges.  A
    // function of the group alone, so results do not depend on timing.
    int pick_cluster(const long long* so, int n) const
    {
        std::vector<int32_t> rel(n + 1);
        for (int p = 0; p <= n; p++) rel[p] = (int32_t)(so[p] - so[0]);
        auto need = [&](int c) {
            size_t m = 0;
            for (int r = 0; r < c; r++) {
                const int a = team_split(rel.data(), n, r, c), b = team_split(rel.data(), n, r + 1, c);
                m = std::max(m, team_layout(n, b - a).need_min);
            }
            return m;
        };
        int c = 0;
        for (int cc = 1; cc <= max_cluster && !c; cc *= 2)
            if (need(cc) <= smem_cap) c = cc;
        while (c && c * 2 <= max_cluster && (long long)rel[n] / c > cta_edges) c *= 2;
        return c;
    }

    // Queued groups start in the order they became ready, each as soon as
    // its CTAs fit under the cap (a later, smaller team may pass a larger
    // one that does not fit yet).  Replaying measured group times through
    // a model of this loop, first-ready-first beat most-edges-first by
    // 10-15 % of the phase: the small groups it held back sat on long chains.
    pg_status pump()
    {
        size_t keep = 0;
        for (size_t k = 0; k < queued.size(); k++) {
            const int t = queued[k];
            if (inflight + tree[t].c <= budget) PG_TRY(launch_group(t));
            else queued[keep++] = t;
        }
        queued.resize(keep);
        return PG_OK;
    }

    pg_status launch_group(int t)
    {
        if (tree[t].stream < 0) PG_TRY(take_stream(&tree[t].stream));
        const Node nd = tree[t];
        cudaStream_t st = ctx->pool[nd.stream];
        if (nd.dep) PG_CUDA(ctx, cudaStreamWaitEvent(st, nd.dep, 0));
        inflight += nd.c;
        const Inputs& in = nd.in;
        uint16_t* sl = nd.sl;
        const int* gl = iota + nd.gi;
        if (nd.c == 1) {
            k_solo<<<1, TEAM_THREADS, smem_cap, st>>>(gl, in, (int)smem_cap, sl);
        } else {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = nd.c;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)nd.c);
            cfg.blockDim = dim3(TEAM_THREADS);
            cfg.dynamicSmemBytes = smem_cap;
            cfg.stream = st;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_clu, gl, in, (int)smem_cap, sl));
        }
        PG_LAUNCHED(ctx);
        running.push_back(t);
        return PG_OK;
    }

    // Group t has ended: decide it as Sub_Partition does and, on a split,
    // start building the children (members partitioned stably by the sign
    // rule of the relabelling, Modularity_CPU.cpp:126-151).
    pg_status finish(int t)
    {
        inflight -= tree[t].c;
        std::memcpy(tree[t].out, hout + (size_t)OUT_W * t, sizeof tree[t].out);
        const double* o = tree[t].out;
        const long long subP = (long long)o[5], subN = (long long)o[6];
        tree[t].split = o[0] > LAMBDA && subP > 1 && subN > 1;
        if (!tree[t].split) {
            free_streams.push_back(tree[t].stream);
            return PG_OK;
        }
        const double coef = (double)(subP - subN) + 0.5;
        const int s = tree[t].s, n = tree[t].n;
        std::vector<int32_t> second;
        int nA = 0;
        long long degA = 0, degB = 0;
        for (int p = 0; p < n; p++) {
            const int32_t id = hAD[s + p];
            const long long d = hR[id + 1] - hR[id];
            if (hv[s + p] * coef > 0.0) {
                hAD[s + nA++] = id;
                degA += d;
            } else {
                second.push_back(id);
                degB += d;
            }
        }
        for (int p = 0; p < n; p++) hgidx[s + p] = p < nA ? 0 : 1;
        std::memcpy(hAD + s + nA, second.data(), sizeof(int32_t) * second.size());
        const size_t b4 = 4 * batches.size();   // the batch's own offsets (read by its teams when they start)
        hgoff[b4] = 0;
        hgoff[b4 + 1] = nA;
        hgoff[b4 + 2] = n;
        hinner[s] = degA;
        hinner[s + 1] = degB;
        const int first = (int)tree.size();
        Node a, b;
        a.s = s;
        a.n = nA;
        b.s = s + nA;
        b.n = n - nA;
        a.parent = b.parent = t;
        tree[t].child = first;
        tree.push_back(a);
        tree.push_back(b);
        Batch bt{s, n, nA, first, tree[t].stream, tree[t].es};
        const int bi = (int)batches.size();
        batches.push_back(bt);
        cudaStream_t st = ctx->pool[bt.stream];
        PG_CUDA(ctx, cudaMemcpyAsync(AD + s, hAD + s, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        PG_CUDA(ctx, cudaMemcpyAsync(gidx + s, hgidx + s, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        PG_CUDA(ctx, cudaMemcpyAsync(agoff + b4, hgoff + b4, 3 * sizeof(long long),
                                     cudaMemcpyHostToDevice, st));
        PG_CUDA(ctx, cudaMemcpyAsync(ainner + s, hinner + s, 2 * sizeof(long long), cudaMemcpyHostToDevice, st));
        const int blocks = std::max(1, std::min((n + 255) / 256, ctx->sm_count));
        k_nm_gprep<<<blocks, 256, 0, st>>>(AD + s, gidx + s, agoff + b4, n, lo + first, label, pos);
        PG_LAUNCHED(ctx);
        const int wblocks = std::max(1, std::min((n + 7) / 8, ctx->sm_count * 4));
        k_nm_gdeg<<<wblocks, 256, 0, st>>>(g->R, g->C, label, AD + s, n, kg + s);
        PG_LAUNCHED(ctx);
        k_nm_gscan<<<1, 1024, 0, st>>>(kg + s, n, asoff + 2 * (size_t)s, dhsoff + 2 * (size_t)s, dhready + bi);
        PG_LAUNCHED(ctx);
        waiting.push_back(bi);
        return PG_OK;
    }

    // The children's in-group degrees are known: fill their sub-graphs and
    // launch both power iterations.
    pg_status start_batch(int bi)
    {
        const Batch bt = batches[bi];
        const size_t s = bt.s, s2 = 2 * s;
        const long long* so = hsoff + s2;
        const long long EA = so[bt.nA], EB = so[bt.P] - so[bt.nA];
        const size_t b4 = 4 * (size_t)bi;
        heoff[b4] = 0;
        heoff[b4 + 1] = EA;
        heoff[b4 + 2] = EA + EB;
        Node& a = tree[bt.first];
        Node& b = tree[bt.first + 1];
        a.es = bt.es;
        a.E = EA;
        b.es = bt.es + EA;
        b.E = EB;
        a.c = pick_cluster(so, bt.nA);
        b.c = pick_cluster(so + bt.nA, bt.P - bt.nA);
        if (!a.c || !b.c) {
            no_fit = true;
            return pg_fail(ctx, PG_ERR_INTERNAL, "modularity: a child group does not fit a team");
        }
        cudaStream_t st = ctx->pool[bt.stream];
        PG_CUDA(ctx, cudaMemcpyAsync(aeoff + b4, heoff + b4, 3 * sizeof(long long), cudaMemcpyHostToDevice, st));
        const int wblocks = std::max(1, std::min((bt.P + 7) / 8, ctx->sm_count * 4));
        k_nm_gfill<<<wblocks, 256, 0, st>>>(g->R, g->C, label, pos, AD + s, bt.P, asoff + s2, agoff + b4, aeoff + b4,
                                            gidx + s, sR + s2, sC + bt.es);
        PG_LAUNCHED(ctx);
        const int blocks = std::max(1, std::min((bt.P + 255) / 256, ctx->sm_count));
        k_nm_gsumbg<<<blocks, 256, 0, st>>>(g->R, AD + s, kg + s, gidx + s, ainner + s, bt.P, base.M, sumBG + s,
                                            kdeg + s);
        PG_LAUNCHED(ctx);
        cudaEvent_t ev;
        PG_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        events.push_back(ev);
        PG_CUDA(ctx, cudaEventRecord(ev, st));
        Inputs in = base;
        in.goff = agoff + b4;
        in.eoff = aeoff + b4;
        in.AD = AD + s;
        in.sR = sR + s2;
        in.sC = sC + bt.es;
        in.kdeg = kdeg + s;
        in.sumBG = sumBG + s;
        in.v = v + s;
        in.v0 = v0 + s;
        in.out = aout + (size_t)OUT_W * bt.first;
        in.hout = dhout + (size_t)OUT_W * bt.first;
        in.hv = dhv + s;
        in.hdone = dhdone + bt.first;
        uint16_t* sl = slices + 2 * bt.es + 64 * (long long)s;
        for (int k = 0; k < 2; k++) {
            Node& nd = tree[bt.first + k];
            nd.in = in;
            nd.gi = k;
            nd.sl = sl;
            nd.stream = k == 0 ? bt.stream : -1;   // the first child runs behind its sub-graph's kernels
            nd.dep = k == 0 ? nullptr : ev;
            queued.push_back(bt.first + k);
        }
        return PG_OK;
    }

    pg_status loop()
    {
        // a flag that never rises (a failed kernel) must not spin forever:
        // while nothing moves, the streams of the running teams are queried
        // now and then, and 120 s without progress is an error
        auto last = std::chrono::steady_clock::now();
        long long idle = 0;
        while (!running.empty() || !waiting.empty() || !queued.empty()) {
            PG_TRY(pump());
            bool any = false;
            for (size_t i = 0; i < running.size();) {
                const int t = running[i];
                if (__atomic_load_n(&hdone[t], __ATOMIC_ACQUIRE)) {
                    running[i] = running.back();
                    running.pop_back();
                    PG_TRY(finish(t));
                    any = true;
                } else {
                    i++;
                }
            }
            for (size_t i = 0; i < waiting.size();) {
                const int bi = waiting[i];
                if (__atomic_load_n(&hready[bi], __ATOMIC_ACQUIRE)) {
                    waiting[i] = waiting.back();
                    waiting.pop_back();
                    PG_TRY(start_batch(bi));
                    any = true;
                } else {
                    i++;
                }
            }
            if (any) {
                idle = 0;
                last = std::chrono::steady_clock::now();
                continue;
            }
            if (++idle % 4096 == 0) {
                for (int t : running) {
                    const cudaError_t e = cudaStreamQuery(ctx->pool[tree[t].stream]);
                    if (e != cudaSuccess && e != cudaErrorNotReady)
                        return pg_fail(ctx, PG_ERR_CUDA, "modularity: team of group %d: %s", t, cudaGetErrorString(e));
                }
                cudaGetLastError();   // not-ready answers are not errors
                if (std::chrono::steady_clock::now() - last > std::chrono::seconds(120))
                    return pg_fail(ctx, PG_ERR_TIMEOUT, "modularity: no team ended for 120 s");
            }
            std::this_thread::yield();
        }
        return PG_OK;
    }

    // Runs the tree below the initial groups to the end; on an error waits
    // for the work in flight (its host functions write into this object).
    pg_status run()
    {
        pg_status st = loop();
        const cudaError_t e = cudaDeviceSynchronize();
        for (cudaEvent_t ev : events) cudaEventDestroy(ev);
        events.clear();
        if (st != PG_OK) return st;
        if (e != cudaSuccess)
            return pg_fail(ctx, PG_ERR_CUDA, "modularity: dependency-driven phase: %s", cudaGetErrorString(e));
        return PG_OK;
    }
};
}  // namespace

// The partition of pg_newman; wv (device, wn values) is the weighted tool's
// value array, null for the unweighted tool.
static pg_status newman_run(pg_ctx* ctx, const pg_graph* g, const float* wv, long long wn, int32_t gpu_rule_above,
                            int32_t* labels, double* Q, int32_t* n_modules, pg_log_fn log, void* user, bool early_ok,
                            bool* retry)
{
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    // log lines are handed to `log` when the call succeeds, so that a call
    // run again (see pg_newman) reports every round once
    std::vector<std::string> lines;
    auto emit = [&](const char* l) { lines.emplace_back(l); };
    const bool weighted = wv != nullptr;
    auto k_coop = weighted ? k_nm_coop<true> : k_nm_coop<false>;
    auto k_grid = weighted ? k_nm_grid<true> : k_nm_grid<false>;
    auto k_solo = weighted ? k_nm_team<SoloTeam, true> : k_nm_team<SoloTeam, false>;
    auto k_clu = weighted ? k_nm_team<ClusterTeam, true> : k_nm_team<ClusterTeam, false>;
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
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coop, COOP_THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "power iteration kernel cannot be resident");
    const int coop_grid = ctx->sm_count;   // one fat block per SM keeps the grid barrier short
    PG_TRY(pg_wst(ctx, "nm.part", (size_t)coop_grid * 8 + 8, &part));
    uint16_t* c16;
    PG_TRY(pg_wst(ctx, "nm.c16", (size_t)nnz + 8, &c16));
    uint16_t* slices;   // team CTAs whose sliced rows do not fit shared memory
    PG_TRY(pg_wst(ctx, "nm.slices", (size_t)2 * nnz + 64 * (size_t)n + 64, &slices));
    PG_TRY(pg_wst(ctx, "nm.sR", 2 * (size_t)n + 4, &sR));   // n+1 offsets per group at twice its first member
    // dependency-driven phase: every buffer is taken here, before any of its
    // streams runs (growing a buffer later would free it under them)
    NmAsync as;
    const size_t max_nodes = 2 * (size_t)n + 4;   // tree nodes of the phase (initial groups and children)
    PG_TRY(pg_wst(ctx, "nm.agoff", 4 * (size_t)n + 8, &as.agoff));   // 4 per batch (one batch per split)
    PG_TRY(pg_wst(ctx, "nm.aeoff", 4 * (size_t)n + 8, &as.aeoff));
    PG_TRY(pg_wst(ctx, "nm.asoff", 2 * (size_t)n + 4, &as.asoff));
    PG_TRY(pg_wst(ctx, "nm.ainner", (size_t)n + 4, &as.ainner));
    PG_TRY(pg_wst(ctx, "nm.aout", OUT_W * max_nodes, &as.aout));
    PG_TRY(pg_wst(ctx, "nm.iota", (size_t)n + 4, &as.iota));
    PG_TRY(pg_hwst(ctx, "nm.hAD", (size_t)n + 4, &as.hAD));
    PG_TRY(pg_hwst(ctx, "nm.hgidx", (size_t)n + 4, &as.hgidx));
    PG_TRY(pg_hwst(ctx, "nm.hsoff", 2 * (size_t)n + 4, &as.hsoff));
    PG_TRY(pg_hwst(ctx, "nm.hgoff", 4 * (size_t)n + 8, &as.hgoff));
    PG_TRY(pg_hwst(ctx, "nm.heoff", 4 * (size_t)n + 8, &as.heoff));
    PG_TRY(pg_hwst(ctx, "nm.hinner", (size_t)n + 4, &as.hinner));
    PG_TRY(pg_hwst(ctx, "nm.hv", (size_t)n + 4, &as.hv));
    PG_TRY(pg_hwst(ctx, "nm.hout", OUT_W * max_nodes, &as.hout));
    PG_TRY(pg_hwst(ctx, "nm.hdone", max_nodes, &as.hdone));
    PG_TRY(pg_hwst(ctx, "nm.hready", (size_t)n + 4, &as.hready));
    int max_cluster = CLUSTER;  // 16 needs the non-portable opt-in
    if (cudaFuncSetAttribute(k_clu, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        max_cluster = 8;
    }
    for (auto& st : ctx->side)
        if (!st) PG_CUDA(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const size_t smem_cap = std::min(SMEM_CAP, (size_t)ctx->smem_optin - 4096);
    PG_CUDA(ctx, cudaFuncSetAttribute(k_solo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    PG_CUDA(ctx,
            cudaFuncSetAttribute(k_clu, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    PG_CUDA(ctx, cudaFuncSetAttribute(k_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    int grid_per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid_per_sm, k_grid, COOP_THREADS, smem_cap));
    PG_CUDA(ctx, cudaMemsetAsync(label, 0, sizeof(int32_t) * (n + 1), ctx->stream));

    std::vector<int32_t> hR(n + 1), hl(n);
    PG_TRY(pg_d2h(ctx, hR.data(), g->R, sizeof(int32_t) * (n + 1)));
    const int grid = ctx->sm_count * 4;
    // the largest double whose correctly rounded square root is at most
    // EPSILON: the loop test sqrt(e) > EPSILON is e > err_sq
    double err_sq = EPSILON * EPSILON;
    while (std::sqrt(err_sq) > EPSILON) err_sq = std::nextafter(err_sq, 0.0);
    while (std::sqrt(std::nextafter(err_sq, 1.0)) <= EPSILON) err_sq = std::nextafter(err_sq, 1.0);
    std::vector<int32_t> adjust((size_t)n + 2, 0);
    int Round = 0, Max_Result = 0, Module_Num = 1, Index = 1;
    char line[512];
    std::vector<int32_t> hAD(n), hgidx(n), hpos(n, 0);
    // wall time per kind of power-iteration launch, reported in the log
    double t_small = 0, t_large = 0, t_setup = 0, t_async = 0;
    long long it_small = 0, it_large = 0, it_async = 0;
    int generations = 0;
    // dependency-driven phase: device label of tree index 0 (-1: not reached),
    // round of every tree node, labels in use
    int async_lo = -1, label_bound = 0, async_groups = 0, chain_groups = 0;
    double chain_ms = 0.0, span_ms = 0.0, busy_ctas = 0.0;
    std::vector<int> ref_of;
    const long long async_cta_edges = ASYNC_CTA_EDGES;
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
        PG_TRY(pg_wst(ctx, "nm.goff", (size_t)G + 1, &goff));
        PG_TRY(pg_wst(ctx, "nm.eoff", (size_t)G + 1, &eoff));
        PG_TRY(pg_wst(ctx, "nm.inner", (size_t)G, &innerM));
        PG_TRY(pg_wst(ctx, "nm.out", (size_t)G * OUT_W, &out));
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
        in.v = v; in.v0 = v0; in.M = M; in.gpu_rule_above = gpu_rule_above; in.out = out; in.err_sq = err_sq;
        in.wv = wv; in.wn = wn;
        in.hout = nullptr; in.hv = nullptr; in.hdone = nullptr;
        // Shared memory of the largest CTA of group q split over c CTAs,
        // before its sliced columns
        auto team_need = [&](int q, int c) {
            const int ng = (int)(hgoff[q + 1] - hgoff[q]);
            std::vector<int32_t> rel(ng + 1);
            for (int p = 0; p <= ng; p++) rel[p] = (int32_t)(hsoff[hgoff[q] + p] - heoff[q]);
            size_t need = 0;
            for (int r = 0; r < c; r++) {
                const int a = team_split(rel.data(), ng, r, c), b = team_split(rel.data(), ng, r + 1, c);
                need = std::max(need, team_layout(ng, b - a).need_min);
            }
            return need;
        };
        // groups by size: teams (one cluster of 1-16 CTAs each), the rest on
        // the whole grid
        std::vector<int> team, large;
        std::vector<int> csz;
        for (int q = 0; q < G; q++) {
            const long long ng = hgoff[q + 1] - hgoff[q];
            if (ng == 0) continue;
            const long long edges = heoff[q + 1] - heoff[q];
            int c = 0;
            if (edges <= MEDIUM_EDGES && ng <= TEAM_MAX_ROWS)
                for (int cc = 1; cc <= max_cluster && !c; cc *= 2)
                    if (team_need(q, cc) <= smem_cap) c = cc;
            if (c) {
                team.push_back(q);
                csz.push_back(c);
            } else {
                large.push_back(q);
            }
        }
        // SMs: double the team with the most edges per CTA while SMs are
        // left and each CTA keeps at least MIN_CTA_EDGES edges
        {
            int used = 0;
            for (int c : csz) used += c;
            const int budget = std::max(ctx->sm_count, used);
            for (;;) {
                int best = -1;
                double best_load = 0.0;
                for (size_t j = 0; j < team.size(); j++) {
                    const long long e = heoff[team[j] + 1] - heoff[team[j]];
                    const double load = (double)e / csz[j];
                    if (csz[j] * 2 <= max_cluster && load >= 2.0 * MIN_CTA_EDGES && load > best_load) {
                        best = (int)j;
                        best_load = load;
                    }
                }
                if (best < 0 || used + csz[best] > budget) break;
                used += csz[best];
                csz[best] *= 2;
            }
        }
        // whole-grid groups first (each needs the whole GPU).  When every
        // child of theirs fits a team, the dependency-driven phase starts
        // right after them and takes this generation's teams along, instead
        // of running those alone and holding every child back until the
        // generation is decided
        std::vector<double> hout((size_t)G * OUT_W, 0.0);
        bool early = false;
        if (!large.empty()) {
            auto t0 = now();
            for (int q : large) {
                int qq = q;
                // column blocks as large as the shared memory of the CTA with the
                // most rows allows; the gather kernel when even 1024 do not fit
                const int ng = (int)(hgoff[q + 1] - hgoff[q]);
                std::vector<int32_t> rel(ng + 1);
                for (int p = 0; p <= ng; p++) rel[p] = (int32_t)(hsoff[hgoff[q] + p] - heoff[q]);
                int most = 0;
                for (int r = 0; r < coop_grid; r++)
                    most = std::max(most, team_split(rel.data(), ng, r + 1, coop_grid) - team_split(rel.data(), ng, r, coop_grid));
                int cb_log = 0;
                for (int lg = 14; lg >= 10 && !cb_log; lg--) {
                    const int nblk = (ng + (1 << lg) - 1) >> lg;
                    if (grid_layout(most, nblk, 1 << lg).need <= smem_cap) cb_log = lg;
                }
                if (cb_log && grid_per_sm >= 1) {
                    const size_t need = grid_layout(most, (ng + (1 << cb_log) - 1) >> cb_log, 1 << cb_log).need;
                    void* args[] = {(void*)&qq, (void*)&in, (void*)&part, (void*)&c16, (void*)&cb_log};
                    PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_grid, dim3(coop_grid), dim3(COOP_THREADS), args,
                                                             need, ctx->stream));
                } else {
                    void* args[] = {(void*)&qq, (void*)&in, (void*)&part};
                    PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_coop, dim3(coop_grid), dim3(COOP_THREADS), args, 0,
                                                             ctx->stream));
                }
                PG_LAUNCHED(ctx);
            }
            PG_TRY(pg_d2h(ctx, hout.data(), out, sizeof(double) * G * OUT_W));
            t_large += ms_since(t0);
            for (int q : large) it_large += (long long)(hout[(size_t)q * OUT_W + 1] + hout[(size_t)q * OUT_W + 3]);
            early = early_ok;
            for (int q : large) {
                const double* o = &hout[(size_t)q * OUT_W];
                const long long subP = (long long)o[5], subN = (long long)o[6];
                if (o[0] > LAMBDA && subP > 1 && subN > 1 && (subP > TEAM_MAX_ROWS || subN > TEAM_MAX_ROWS)) early = false;
            }
        }
        if (large.empty() || early) {
            // ---- every pending group fits a team: dependency-driven from here on
            auto t_as = now();
            as.ctx = ctx;
            as.g = g;
            as.k_solo = k_solo;
            as.k_clu = k_clu;
            as.base = in;
            as.base.out = as.aout;
            as.lo = lo;
            as.smem_cap = smem_cap;
            as.max_cluster = max_cluster;
            as.cta_edges = async_cta_edges;
            as.hR = hR.data();
            as.label = label; as.pos = pos; as.AD = AD; as.gidx = gidx; as.kg = kg; as.sR = sR; as.sC = sC;
            as.v = v; as.v0 = v0; as.sumBG = sumBG; as.kdeg = kdeg; as.slices = slices;
            k_nm_iota<<<ctx->sm_count, 256, 0, ctx->stream>>>(as.iota, n + 4);
            PG_LAUNCHED(ctx);
            PG_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
            std::memcpy(as.hAD, hAD.data(), sizeof(int32_t) * P);
            // streams are created here, with the device idle: creating one
            // while teams run blocked the host for up to ~100 ms
            PG_TRY(pg_stream_pool(ctx, POOL_STREAMS));
            for (int k = (int)ctx->pool.size() - 1; k >= 0; k--) as.free_streams.push_back(k);
            PG_TRY(as.map_pinned());
            std::memset(as.hdone, 0, sizeof(int) * max_nodes);
            std::memset(as.hready, 0, sizeof(int) * ((size_t)n + 4));
            Inputs in0 = in;
            in0.out = as.aout;
            in0.hout = as.dhout;
            in0.hv = as.dhv;
            in0.hdone = as.dhdone;
            for (int q = 0; q < G; q++) {
                NmAsync::Node nd;
                nd.s = (int)hgoff[q];
                nd.n = (int)(hgoff[q + 1] - hgoff[q]);
                nd.es = heoff[q];
                nd.E = heoff[q + 1] - heoff[q];
                as.tree.push_back(nd);
            }
            as.budget = std::max(max_cluster, ctx->sm_count - RESERVE_SMS);
            for (int q : large) {   // already run on the whole grid (early start only)
                NmAsync::Node& nd = as.tree[q];
                nd.c = 0;
                nd.grid = true;
                PG_TRY(as.take_stream(&nd.stream));
                std::memcpy(as.hout + (size_t)OUT_W * q, &hout[(size_t)q * OUT_W], sizeof(double) * OUT_W);
                as.hout[(size_t)OUT_W * q + 8] = as.hout[(size_t)OUT_W * q + 9] = 0.0;   // not a team: no clock
                PG_TRY(pg_d2h(ctx, as.hv + nd.s, v + nd.s, sizeof(double) * nd.n));
                as.hdone[q] = 1;
                as.running.push_back(q);
            }
            for (int q = 0; q < G; q++) {
                NmAsync::Node& nd = as.tree[q];
                if (nd.n == 0 || nd.grid) continue;
                nd.c = as.pick_cluster(&hsoff[hgoff[q]], nd.n);
                if (!nd.c) return pg_fail(ctx, PG_ERR_INTERNAL, "modularity: a group does not fit a team");
                nd.in = in0;
                nd.gi = q;
                nd.sl = slices;
                nd.dep = ctx->ev[0];
                as.queued.push_back(q);
            }
            {
                const pg_status st = as.run();
                if (st != PG_OK) {
                    // a child of a whole-grid group did not fit a team: the
                    // caller runs the call again without the early start
                    if (retry) *retry = as.no_fit && early;
                    return st;
                }
            }
            t_async += ms_since(t_as);
            // ---- the reference's rounds over the finished tree, in order
            std::vector<int> round_tree((size_t)hi + as.tree.size() + 4, -1);
            for (int q = 0; q < G; q++)
                if (as.tree[q].n > 0) round_tree[lo + q] = q;
            ref_of.assign(as.tree.size(), -1);
            for (int round = lo; round <= Max_Result; round++) {
                const int t = round_tree[round];
                if (t < 0) continue;
                ref_of[t] = round;
                const NmAsync::Node& nd = as.tree[t];
                const double* o = nd.out;
                if (!nd.grid) it_async += (long long)(o[1] + o[3]);
                if (log) {
                    int len = snprintf(line, sizeof line, "Round:\t%d\tnumber of nodes:\t%d\tIterations:\t%d\tresidual:\t%g\t",
                                       round, nd.n, (int)o[1], o[2]);
                    if (o[7] != 0.0)
                        len += snprintf(line + len, sizeof line - len, "Iterations:\t%d\tresidual:\t%g\t", (int)o[3], o[4]);
                    snprintf(line + len, sizeof line - len, "Eigen Value: %g\tDivide?: %d", o[0], (int)nd.split);
                    emit(line);
                }
                if (nd.split) {
                    round_tree[Max_Result + 1] = nd.child;
                    round_tree[Max_Result + 2] = nd.child + 1;
                    Max_Result += 2;
                } else {
                    if (round >= (int)adjust.size()) adjust.resize(round + 1, 0);
                    adjust[round] = Index++;
                }
                Module_Num += nd.split;
            }
            // the chain of groups that ended last: its run time against the
            // phase's span shows what waiting for SMs and the host costs
            {
                double t_begin = 1e300, t_end = 0.0, busy = 0.0;
                int last = -1;
                for (size_t t = 0; t < as.tree.size(); t++) {
                    const NmAsync::Node& nd = as.tree[t];
                    if (nd.n == 0 || nd.grid) continue;
                    t_begin = std::min(t_begin, nd.out[8]);
                    if (nd.out[9] > t_end) {
                        t_end = nd.out[9];
                        last = (int)t;
                    }
                    busy += nd.c * (nd.out[9] - nd.out[8]);
                }
                for (int t = last; t >= 0; t = as.tree[t].parent) {
                    chain_groups++;
                    chain_ms += (as.tree[t].out[9] - as.tree[t].out[8]) * 1e-6;
                }
                if (last >= 0) {
                    span_ms = (t_end - t_begin) * 1e-6;
                    busy_ctas = busy / (t_end - t_begin);
                }
            }
            async_lo = lo;
            label_bound = std::max(Max_Result, lo + (int)as.tree.size());
            async_groups = (int)as.tree.size();
            break;
        }
        // glist by cluster size, largest first; one launch per size
        std::vector<int> lists;
        struct Bucket { int c; size_t b, e; size_t smem; };
        std::vector<Bucket> buckets;
        for (int c = max_cluster; c >= 1; c >>= 1) {
            // every CTA gets the whole budget; what its rows leave holds the slices
            Bucket bk{c, lists.size(), 0, smem_cap};
            for (size_t j = 0; j < team.size(); j++)
                if (csz[j] == c) lists.push_back(team[j]);
            bk.e = lists.size();
            if (bk.e > bk.b) buckets.push_back(bk);
        }
        if (!lists.empty())
            PG_CUDA(ctx, cudaMemcpyAsync(glist, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice,
                                         ctx->stream));
        auto t0 = now();
        if (!buckets.empty()) {
            // the launches of a generation run beside each other, one stream each
            PG_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
            int si = 0;
            for (const Bucket& bk : buckets) {
                cudaStream_t st = ctx->side[si++];
                PG_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev[0], 0));
                const int* blist = glist + bk.b;
                const int nbytes = (int)bk.smem;
                if (bk.c == 1) {
                    k_solo<<<(unsigned)(bk.e - bk.b), TEAM_THREADS, bk.smem, st>>>(blist, in, nbytes, slices);
                } else {
                    cudaLaunchConfig_t cfg = {};
                    cudaLaunchAttribute attr[1];
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = bk.c;
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    cfg.gridDim = dim3((unsigned)((bk.e - bk.b) * bk.c));
                    cfg.blockDim = dim3(TEAM_THREADS);
                    cfg.dynamicSmemBytes = bk.smem;
                    cfg.stream = st;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_clu, blist, in, nbytes, slices));
                }
                PG_LAUNCHED(ctx);
            }
            for (int j = 0; j < si; j++) {
                PG_CUDA(ctx, cudaEventRecord(ctx->ev[1 + j], ctx->side[j]));
                PG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev[1 + j], 0));
            }
            PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        t_small += ms_since(t0);
        PG_TRY(pg_d2h(ctx, hout.data(), out, sizeof(double) * G * OUT_W));
        for (int q : team) it_small += (long long)(hout[(size_t)q * OUT_W + 1] + hout[(size_t)q * OUT_W + 3]);
        // ---- decisions in round order (labels exactly as the sequential reference)
        std::vector<int> hbase(G, -1);
        std::vector<double> hcoef(G, 0.0);
        bool any_split = false;
        for (int q = 0; q < G; q++) {
            const int round = lo + q;
            const long long ng = hgoff[q + 1] - hgoff[q];
            if (ng == 0) continue;
            const double* o = &hout[(size_t)q * OUT_W];
            const long long subP = (long long)o[5], subN = (long long)o[6];
            const bool issub = o[0] > LAMBDA && subP > 1 && subN > 1;
            if (log) {
                int len = snprintf(line, sizeof line, "Round:\t%d\tnumber of nodes:\t%lld\tIterations:\t%d\tresidual:\t%g\t",
                                   round, ng, (int)o[1], o[2]);
                if (o[7] != 0.0)
                    len += snprintf(line + len, sizeof line - len, "Iterations:\t%d\tresidual:\t%g\t", (int)o[3], o[4]);
                snprintf(line + len, sizeof line - len, "Eigen Value: %g\tDivide?: %d", o[0], (int)issub);
                emit(line);
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
    label_bound = std::max(label_bound, Max_Result);
    unsigned long long* Kc;
    PG_TRY(pg_wst(ctx, "nm.Kc", (size_t)label_bound + 4, &Kc));
    PG_CUDA(ctx, cudaMemsetAsync(Kc, 0, sizeof(unsigned long long) * (label_bound + 2), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(unsigned long long), ctx->stream));
    k_nm_q<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, n, acc, Kc);
    PG_LAUNCHED(ctx);
    unsigned long long inside = 0;
    std::vector<unsigned long long> K(label_bound + 1);
    PG_TRY(pg_d2h(ctx, &inside, acc, sizeof inside));
    PG_TRY(pg_d2h(ctx, K.data(), Kc, sizeof(unsigned long long) * (label_bound + 1)));
    double sq = 0.0;
    for (int c = 0; c <= label_bound; c++) sq += (double)K[c] * (double)K[c];
    const double q = ((double)inside - sq / 2 / M) / (2.0 * M);
    PG_TRY(pg_d2h(ctx, hl.data(), label, sizeof(int32_t) * n));
    for (int i = 0; i < n; i++) {
        const int l = hl[i];
        labels[i] = adjust[async_lo >= 0 && l >= async_lo ? ref_of[l - async_lo] : l];
    }
    if (Q) *Q = q;
    if (n_modules) *n_modules = Module_Num;
    if (log) {
        snprintf(line, sizeof line, "Number of Modules: %d,\tQ=%.6g", Module_Num, q);
        emit(line);
        snprintf(line, sizeof line,
                 "Timing (ms): generations %d, setup %.1f, team groups %.1f (%lld iterations), "
                 "cooperative groups %.1f (%lld), dependency-driven phase %.1f (%d groups, %lld iterations; "
                 "device span %.1f, last chain %d groups running %.1f, mean team CTAs busy %.1f)",
                 generations, t_setup, t_small, it_small, t_large, it_large, t_async, async_groups, it_async, span_ms,
                 chain_groups, chain_ms, busy_ctas);
        emit(line);
        for (const std::string& l : lines) log(l.c_str(), user);
    }
    return PG_OK;
}

extern "C" pg_status pg_newman(pg_ctx* ctx, const pg_graph* g, int32_t gpu_rule_above, int32_t* labels, double* Q,
                               int32_t* n_modules, pg_log_fn log, void* user)
{
    if (!ctx || !g || !labels) return pg_fail(ctx, PG_ERR_INVALID, "pg_newman: null argument");
    bool retry = false;
    const pg_status st = newman_run(ctx, g, nullptr, 0, gpu_rule_above, labels, Q, n_modules, log, user, true, &retry);
    if (st == PG_OK || !retry) return st;
    return newman_run(ctx, g, nullptr, 0, gpu_rule_above, labels, Q, n_modules, log, user, false, nullptr);
}

extern "C" pg_status pg_newman_weighted(pg_ctx* ctx, const pg_graph* g, const pg_graph* weights_of,
                                        int32_t gpu_rule_above, int32_t* labels, double* Q, int32_t* n_modules,
                                        pg_log_fn log, void* user)
{
    if (!ctx || !g || !labels) return pg_fail(ctx, PG_ERR_INVALID, "pg_newman_weighted: null argument");
    const pg_graph* w = weights_of ? weights_of : g;
    if (!w->V) return pg_fail(ctx, PG_ERR_INVALID, "pg_newman_weighted: the weight graph has no weights");
    if (w->device != g->device) return pg_fail(ctx, PG_ERR_INVALID, "pg_newman_weighted: graphs on different devices");
    bool retry = false;
    const pg_status st = newman_run(ctx, g, w->V, w->nnz, gpu_rule_above, labels, Q, n_modules, log, user, true, &retry);
    if (st == PG_OK || !retry) return st;
    return newman_run(ctx, g, w->V, w->nnz, gpu_rule_above, labels, Q, n_modules, log, user, false, nullptr);
}
