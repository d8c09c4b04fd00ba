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
// afterwards gives exactly the reference's labelling.  Per generation:
//   - induced sub-graphs of all groups at once (columns keep original ids,
//     as the reference's NewCol);
//   - groups with few edges: one CTA per group runs the whole power
//     iteration (block barriers only), all such groups in one launch;
//   - large groups: one cooperative kernel per group, the three reductions
//     per iteration separated by grid-wide barriers.
// Reductions are FP64 in a fixed order: results are deterministic.
#include "pg_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>

namespace cg = cooperative_groups;

namespace {
constexpr int THREADS = 256;
constexpr int MAX_ITER = 10000;
constexpr double EPSILON = 1e-6;
constexpr double LAMBDA = 0.01;
constexpr long long SMALL_EDGES = 1LL << 15;   // at most this many edges: one CTA per group
constexpr long long MEDIUM_EDGES = 1LL << 22;  // at most this many edges: one cluster per group
constexpr int CLUSTER = 16;                    // CTAs per cluster for medium groups

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

// Induced CSR rows (columns keep original node ids and CSR order).
__global__ void k_nm_gfill(const int32_t* __restrict__ R, const int32_t* __restrict__ C,
                           const int32_t* __restrict__ label, const int32_t* __restrict__ AD, int32_t P,
                           const long long* __restrict__ soff, int32_t* __restrict__ sR, int32_t* __restrict__ sC)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = gw; p < P; p += nw) {
        int i = AD[p], li = label[i];
        long long pos = soff[p];
        if (lane == 0) {
            sR[p] = (int32_t)pos;
            if (p == P - 1) sR[P] = (int32_t)soff[P];
        }
        for (int32_t base = R[i]; base < R[i + 1]; base += 32) {
            int32_t q = base + lane;
            bool in = q < R[i + 1] && label[C[q]] == li;
            unsigned m = __ballot_sync(0xffffffffu, in);
            if (in) sC[pos + __popc(m & ((1u << lane) - 1u))] = C[q];
            pos += __popc(m);
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

// Sum over the block, result returned to every thread.
__device__ double block_allsum(double x, double* sh)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < nw; q++) t += sh[q];
        sh[32] = t;
    }
    __syncthreads();
    return sh[32];
}

struct Group {
    const int32_t* AD;
    const int32_t* sR;      // row offsets into sC (global positions)
    const int32_t* sC;
    const double* kdeg;
    const double* sumBG;
    double* v;
    double* v0;
    int ng;
};

// Reduction across the CTAs of a thread-block cluster through distributed
// shared memory: every CTA publishes its block sum in slot[par][k], the
// cluster barrier orders it, and each CTA adds the published values in rank
// order (the same order everywhere, so every CTA holds the same total).
struct ClusterReduce {
    double slot[2][4];
    double bcast[4];
};

__device__ void cluster_sums(cg::cluster_group& cl, ClusterReduce* cr, int par, const double* x, int k, double* out,
                             double* sh)
{
    for (int q = 0; q < k; q++) {
        double t = block_allsum(x[q], sh);
        if (threadIdx.x == 0) cr->slot[par][q] = t;
    }
    __threadfence();
    cl.sync();
    if (threadIdx.x == 0) {
        const int nb = (int)cl.num_blocks();
        for (int q = 0; q < k; q++) {
            double t = 0.0;
            for (int r = 0; r < nb; r++) t += cl.map_shared_rank(cr, r)->slot[par][q];
            cr->bcast[q] = t;
        }
    }
    __syncthreads();
    for (int q = 0; q < k; q++) out[q] = cr->bcast[q];
    __syncthreads();
}

// Lead_Vector on one cluster (a cluster of one CTA is a single block);
// returns lambda and fills iterations / residual.
__device__ double lead_vector_cluster(const Group& g, double* vv, int M, double beta, int* iters, double* resid,
                                      double* sh, ClusterReduce* cr, int& par)
{
    cg::cluster_group cl = cg::this_cluster();
    const int B = blockDim.x;
    const int ct = (int)cl.block_rank() * B + threadIdx.x, cth = (int)cl.num_blocks() * B;
    const int lane = threadIdx.x & 31, cw = ct >> 5, cnw = cth >> 5;
    for (int p = ct; p < g.ng; p += cth) g.v[p] = (double)g.AD[p];
    __threadfence();
    cl.sync();
    double err1 = 1.0, err2 = 1.0, vnorm = 0.0;
    int iter = 0;
    double in[2], out[2];
    while (err1 > EPSILON && err2 > EPSILON && iter < MAX_ITER) {
        double x = 0.0;
        for (int p = ct; p < g.ng; p += cth) {
            double vp = g.v[p];
            g.v0[p] = vp;
            vv[g.AD[p]] = vp;
            x += vp * g.kdeg[p];
        }
        in[0] = x;
        cluster_sums(cl, cr, par, in, 1, out, sh);
        par ^= 1;
        const double c = out[0] / 2.0 / (double)M;
        double y2 = 0.0;
        for (int p = cw; p < g.ng; p += cnw) {
            double s = 0.0;
            for (int32_t q = g.sR[p] + lane; q < g.sR[p + 1]; q += 32) s += vv[g.sC[q]];
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) {
                s -= c * g.kdeg[p] + (g.sumBG[p] - beta) * g.v0[p];
                g.v[p] = s;
                y2 += s * s;
            }
        }
        in[0] = y2;
        cluster_sums(cl, cr, par, in, 1, out, sh);
        par ^= 1;
        vnorm = sqrt(out[0]);
        double e1 = 0.0, e2 = 0.0;
        for (int p = ct; p < g.ng; p += cth) {
            double vp = g.v[p] / vnorm;
            g.v[p] = vp;
            double d1 = vp - g.v0[p], d2 = vp + g.v0[p];
            e1 += d1 * d1;
            e2 += d2 * d2;
        }
        in[0] = e1;
        in[1] = e2;
        cluster_sums(cl, cr, par, in, 2, out, sh);
        par ^= 1;
        err1 = sqrt(out[0]);
        err2 = sqrt(out[1]);
        iter++;
    }
    // first entry of largest magnitude decides the sign (Modularity_CPU.cpp:291-296):
    // per CTA (value, index), then the CTAs in rank order.
    double best = -1.0;
    int bi = 0x7fffffff;
    for (int p = ct; p < g.ng; p += cth) {
        double m = fabs(g.v[p]);
        if (m > best) { best = m; bi = p; }
    }
    for (int o = 16; o; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    __shared__ double sb[32];
    __shared__ int si[32];
    __syncthreads();
    if (lane == 0) { sb[threadIdx.x >> 5] = best; si[threadIdx.x >> 5] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1.0;
        int ix = 0x7fffffff;
        for (int q = 0; q < (B >> 5); q++)
            if (sb[q] > b || (sb[q] == b && si[q] < ix)) { b = sb[q]; ix = si[q]; }
        cr->slot[par][0] = b;
        cr->slot[par][1] = (double)ix;
    }
    __threadfence();
    cl.sync();
    if (threadIdx.x == 0) {
        double b = -1.0;
        int ix = 0x7fffffff;
        for (int r = 0; r < (int)cl.num_blocks(); r++) {
            const ClusterReduce* o = cl.map_shared_rank(cr, r);
            double ob = o->slot[par][0];
            int oi = (int)o->slot[par][1];
            if (ob > b || (ob == b && oi < ix)) { b = ob; ix = oi; }
        }
        si[0] = ix;
    }
    par ^= 1;
    __syncthreads();
    const int mx = si[0];
    *iters = iter;
    *resid = fmin(err1, err2);
    double lam = 0.0;
    if (g.ng > 0) lam = (g.v[mx] * g.v0[mx] > 0) ? vnorm : -vnorm;
    __syncthreads();
    return lam;
}

// One group per cluster (cluster size 1 for small groups, up to 16 CTAs for
// medium ones).  out per group: lambda, it0, res0, it1, res1, subP, subN, shifted.
__global__ void __launch_bounds__(THREADS)
k_nm_cluster(const int* __restrict__ glist, const long long* __restrict__ goff, const int32_t* __restrict__ AD,
             const int32_t* __restrict__ sR, const int32_t* __restrict__ sC, const double* __restrict__ kdeg,
             const double* __restrict__ sumBG, double* __restrict__ v, double* __restrict__ v0,
             double* __restrict__ vv, int M, int gpu_rule_above, double* __restrict__ out)
{
    __shared__ double sh[40];
    __shared__ ClusterReduce cr;
    cg::cluster_group cl = cg::this_cluster();
    const int gi = glist[blockIdx.x / cl.num_blocks()];
    const long long p0 = goff[gi];
    Group g;
    g.ng = (int)(goff[gi + 1] - p0);
    g.AD = AD + p0; g.sR = sR + p0; g.sC = sC; g.kdeg = kdeg + p0; g.sumBG = sumBG + p0;
    g.v = v + p0; g.v0 = v0 + p0;
    int par = 0;
    int it0, it1 = 0;
    double r0, r1 = 0.0;
    double lam = lead_vector_cluster(g, vv, M, 0.0, &it0, &r0, sh, &cr, par);
    const double below = g.ng > gpu_rule_above ? -LAMBDA : 0.0;
    const bool shifted = lam < below;
    if (shifted) lam += lead_vector_cluster(g, vv, M, -lam, &it1, &r1, sh, &cr, par);
    const int ct = (int)cl.block_rank() * blockDim.x + threadIdx.x, cth = (int)cl.num_blocks() * blockDim.x;
    double in[2] = {0.0, 0.0}, res[2];
    for (int p = ct; p < g.ng; p += cth) {
        in[0] += g.v[p] > 0.0;
        in[1] += g.v[p] <= 0.0;
    }
    cluster_sums(cl, &cr, par, in, 2, res, sh);
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
        double* o = out + (size_t)gi * 8;
        o[0] = lam; o[1] = it0; o[2] = r0; o[3] = it1; o[4] = r1; o[5] = res[0]; o[6] = res[1]; o[7] = shifted;
    }
    // no CTA may exit while another still reads its shared memory
    cl.sync();
}

// ---- large groups: cooperative kernel, one group, one pass (beta given)
struct LVArgs {
    Group g;
    int M;
    double beta;
    double* vv;
    double* part;   // [grid][4]
    double* out;    // lambda, iterations, residual, subP, subN
};

__device__ double grid_total(const double* part, int col, double* sh)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) t += part[b * 4 + col];
        sh[33] = t;
    }
    __syncthreads();
    return sh[33];
}

__device__ double block_sum0(double x, double* sh)
{
    return block_allsum(x, sh);
}

__global__ void __launch_bounds__(THREADS) k_nm_coop(LVArgs a)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ double sh[40];
    const Group& g = a.g;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int gw = tid >> 5, nw = nthr >> 5;
    for (int p = tid; p < g.ng; p += nthr) g.v[p] = (double)g.AD[p];
    grid.sync();
    double err1 = 1.0, err2 = 1.0, vnorm = 0.0;
    int iter = 0;
    while (err1 > EPSILON && err2 > EPSILON && iter < MAX_ITER) {
        double x = 0.0;
        for (int p = tid; p < g.ng; p += nthr) {
            double vp = g.v[p];
            g.v0[p] = vp;
            a.vv[g.AD[p]] = vp;
            x += vp * g.kdeg[p];
        }
        double bs = block_sum0(x, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 0] = bs;
        grid.sync();
        const double c = grid_total(a.part, 0, sh) / 2.0 / (double)a.M;
        double y2 = 0.0;
        for (int p = gw; p < g.ng; p += nw) {
            double s = 0.0;
            for (int32_t q = g.sR[p] + lane; q < g.sR[p + 1]; q += 32) s += a.vv[g.sC[q]];
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) {
                s -= c * g.kdeg[p] + (g.sumBG[p] - a.beta) * g.v0[p];
                g.v[p] = s;
                y2 += s * s;
            }
        }
        bs = block_sum0(y2, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 1] = bs;
        grid.sync();
        vnorm = sqrt(grid_total(a.part, 1, sh));
        double e1 = 0.0, e2 = 0.0;
        for (int p = tid; p < g.ng; p += nthr) {
            double vp = g.v[p] / vnorm;
            g.v[p] = vp;
            double d1 = vp - g.v0[p], d2 = vp + g.v0[p];
            e1 += d1 * d1;
            e2 += d2 * d2;
        }
        bs = block_sum0(e1, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 2] = bs;
        bs = block_sum0(e2, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 3] = bs;
        grid.sync();
        err1 = sqrt(grid_total(a.part, 2, sh));
        err2 = sqrt(grid_total(a.part, 3, sh));
        iter++;
        grid.sync();
    }
    if (blockIdx.x == 0) {
        double best = -1.0;
        int bi = 0x7fffffff;
        double sp = 0.0, sn = 0.0;
        for (int p = threadIdx.x; p < g.ng; p += blockDim.x) {
            double m = fabs(g.v[p]);
            if (m > best) { best = m; bi = p; }
            sp += g.v[p] > 0.0;
            sn += g.v[p] <= 0.0;
        }
        for (int o = 16; o; o >>= 1) {
            double ob = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        __shared__ double sb[32];
        __shared__ int si[32];
        const int w = threadIdx.x >> 5, nwb = blockDim.x >> 5;
        if (lane == 0) { sb[w] = best; si[w] = bi; }
        sp = block_allsum(sp, sh);
        sn = block_allsum(sn, sh);
        if (threadIdx.x == 0) {
            double b = -1.0;
            int ix = 0;
            for (int q = 0; q < nwb; q++)
                if (sb[q] > b || (sb[q] == b && si[q] < ix)) { b = sb[q]; ix = si[q]; }
            a.out[0] = g.ng > 0 ? ((g.v[ix] * g.v0[ix] > 0) ? vnorm : -vnorm) : 0.0;
            a.out[1] = iter;
            a.out[2] = fmin(err1, err2);
            a.out[3] = sp;
            a.out[4] = sn;
        }
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
    int32_t *label, *AD, *gidx, *kg, *sR, *sC, *dbase, *glist;
    long long *soff, *goff, *innerM;
    double *v, *v0, *vv, *sumBG, *kdeg, *part, *out, *dcoef;
    unsigned long long* acc;
    PG_TRY(pg_wst(ctx, "nm.label", (size_t)n + 1, &label));
    PG_TRY(pg_wst(ctx, "nm.AD", (size_t)n + 1, &AD));
    PG_TRY(pg_wst(ctx, "nm.gidx", (size_t)n + 1, &gidx));
    PG_TRY(pg_wst(ctx, "nm.kg", (size_t)n + 1, &kg));
    PG_TRY(pg_wst(ctx, "nm.soff", (size_t)n + 2, &soff));
    PG_TRY(pg_wst(ctx, "nm.sR", (size_t)n + 2, &sR));
    PG_TRY(pg_wst(ctx, "nm.sC", (size_t)nnz + 1, &sC));
    PG_TRY(pg_wst(ctx, "nm.v", (size_t)n + 1, &v));
    PG_TRY(pg_wst(ctx, "nm.v0", (size_t)n + 1, &v0));
    PG_TRY(pg_wst(ctx, "nm.vv", (size_t)n + 1, &vv));
    PG_TRY(pg_wst(ctx, "nm.sumBG", (size_t)n + 1, &sumBG));
    PG_TRY(pg_wst(ctx, "nm.kdeg", (size_t)n + 1, &kdeg));
    PG_TRY(pg_wst(ctx, "nm.acc", 4, &acc));
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nm_coop, THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "power iteration kernel cannot be resident");
    const int coop_grid = per_sm * ctx->sm_count;
    // widest cluster the device accepts for the medium-group kernel (16 needs the non-portable opt-in)
    int cluster = CLUSTER;
    if (cudaFuncSetAttribute(k_nm_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        cluster = 8;
    }
    PG_TRY(pg_wst(ctx, "nm.part", (size_t)coop_grid * 4 + 4, &part));
    PG_CUDA(ctx, cudaMemsetAsync(label, 0, sizeof(int32_t) * (n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(vv, 0, sizeof(double) * (n + 1), ctx->stream));

    std::vector<int32_t> hR(n + 1), hl(n);
    PG_TRY(pg_d2h(ctx, hR.data(), g->R, sizeof(int32_t) * (n + 1)));
    const int grid = ctx->sm_count * 4;
    std::vector<int32_t> adjust((size_t)n + 2, 0);
    int Round = 0, Max_Result = 0, Module_Num = 1, Index = 1;
    char line[512];
    std::vector<int32_t> hAD(n), hgidx(n);
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
                    cur[q]++;
                    hinner[q] += hR[i + 1] - hR[i];
                }
        }
        if (P == 0) { Round = hi + 1; continue; }
        PG_TRY(pg_wst(ctx, "nm.goff", (size_t)G + 1, &goff));
        PG_TRY(pg_wst(ctx, "nm.inner", (size_t)G, &innerM));
        PG_TRY(pg_wst(ctx, "nm.out", (size_t)G * 8, &out));
        PG_TRY(pg_wst(ctx, "nm.glist", (size_t)G, &glist));
        PG_TRY(pg_wst(ctx, "nm.base", (size_t)G, &dbase));
        PG_TRY(pg_wst(ctx, "nm.coef", (size_t)G, &dcoef));
        PG_CUDA(ctx, cudaMemcpyAsync(AD, hAD.data(), sizeof(int32_t) * P, cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(gidx, hgidx.data(), sizeof(int32_t) * P, cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(goff, hgoff.data(), sizeof(long long) * (G + 1), cudaMemcpyHostToDevice, ctx->stream));
        PG_CUDA(ctx, cudaMemcpyAsync(innerM, hinner.data(), sizeof(long long) * G, cudaMemcpyHostToDevice, ctx->stream));
        k_nm_gdeg<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, AD, P, kg);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_scan_counts(ctx, kg, (int64_t*)soff, P));
        k_nm_gfill<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, label, AD, P, soff, sR, sC);
        PG_LAUNCHED(ctx);
        k_nm_gsumbg<<<grid, 256, 0, ctx->stream>>>(g->R, AD, kg, gidx, innerM, P, M, sumBG, kdeg);
        PG_LAUNCHED(ctx);
        std::vector<long long> hsoff(P + 1);
        PG_TRY(pg_d2h(ctx, hsoff.data(), soff, sizeof(long long) * (P + 1)));
        t_setup += ms_since(t_gen);
        // ---- power iterations
        std::vector<int> small, medium, large;
        for (int q = 0; q < G; q++) {
            long long ng = hgoff[q + 1] - hgoff[q];
            if (ng == 0) continue;
            long long edges = hsoff[hgoff[q + 1]] - hsoff[hgoff[q]];
            if (edges <= SMALL_EDGES) small.push_back(q);
            else if (edges <= MEDIUM_EDGES && cluster > 1) medium.push_back(q);
            else large.push_back(q);
        }
        std::vector<double> hout((size_t)G * 8, 0.0);
        if (!small.empty() || !medium.empty()) {
            std::vector<int> lists(small);
            lists.insert(lists.end(), medium.begin(), medium.end());
            PG_CUDA(ctx, cudaMemcpyAsync(glist, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice,
                                         ctx->stream));
            if (!small.empty()) {
                auto t0 = now();
                k_nm_cluster<<<(int)small.size(), THREADS, 0, ctx->stream>>>(glist, goff, AD, sR, sC, kdeg, sumBG, v,
                                                                             v0, vv, M, gpu_rule_above, out);
                PG_LAUNCHED(ctx);
                PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
                t_small += ms_since(t0);
            }
            if (!medium.empty()) {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = cluster;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3((unsigned)(medium.size() * cluster));
                cfg.blockDim = dim3(THREADS);
                cfg.stream = ctx->stream;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                const int* mlist = glist + small.size();
                auto t0 = now();
                PG_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_nm_cluster, mlist, (const long long*)goff, (const int32_t*)AD,
                                                (const int32_t*)sR, (const int32_t*)sC, (const double*)kdeg,
                                                (const double*)sumBG, v, v0, vv, M, (int)gpu_rule_above, out));
                PG_LAUNCHED(ctx);
                PG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
                t_medium += ms_since(t0);
            }
            PG_TRY(pg_d2h(ctx, hout.data(), out, sizeof(double) * G * 8));
            for (int q : small) it_small += (long long)(hout[(size_t)q * 8 + 1] + hout[(size_t)q * 8 + 3]);
            for (int q : medium) it_medium += (long long)(hout[(size_t)q * 8 + 1] + hout[(size_t)q * 8 + 3]);
        }
        auto t_l = now();
        for (int q : large) {
            const long long p0 = hgoff[q];
            LVArgs a;
            a.g.ng = (int)(hgoff[q + 1] - p0);
            a.g.AD = AD + p0; a.g.sR = sR + p0; a.g.sC = sC; a.g.kdeg = kdeg + p0; a.g.sumBG = sumBG + p0;
            a.g.v = v + p0; a.g.v0 = v0 + p0;
            a.M = M; a.beta = 0.0; a.vv = vv; a.part = part; a.out = out + (size_t)q * 8;
            double r[2][5];
            bool shifted = false;
            for (int pass = 0; pass < 2; pass++) {
                void* args[] = {(void*)&a};
                PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_nm_coop, dim3(coop_grid), dim3(THREADS), args, 0,
                                                         ctx->stream));
                PG_LAUNCHED(ctx);
                PG_TRY(pg_d2h(ctx, r[pass], a.out, sizeof(double) * 5));
                if (pass == 0) {
                    const double below = a.g.ng > gpu_rule_above ? -LAMBDA : 0.0;
                    if (!(r[0][0] < below)) break;
                    shifted = true;
                    a.beta = -r[0][0];
                }
            }
            double* o = &hout[(size_t)q * 8];
            o[0] = shifted ? r[0][0] + r[1][0] : r[0][0];
            o[1] = r[0][1]; o[2] = r[0][2];
            o[3] = shifted ? r[1][1] : 0; o[4] = shifted ? r[1][2] : 0;
            o[5] = shifted ? r[1][3] : r[0][3];
            o[6] = shifted ? r[1][4] : r[0][4];
            o[7] = shifted;
            it_large += (long long)(o[1] + o[3]);
        }
        t_large += ms_since(t_l);
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
