// newman.cu -- Newman leading-eigenvector modularity (Partition_GPU /
// Sub_Partition_GPU / Lead_Vector_GPU, U/cuda_EC/cuda_EC/modularity_GPU.cu:230-530;
// CPU twins Partition / Sub_Partition / Lead_Vector, Modularity_CPU.cpp:48-298).
//
// Rounds follow the reference: round r takes the nodes labelled r, builds
// the induced sub-graph, finds the leading eigenvector of the generalised
// modularity matrix B(g) - diag(sumBG) by power iteration from v = node ids
// (tolerance 1e-6 on |v - v0| or |v + v0|, at most 10,000 iterations,
// shifted rerun when the eigenvalue is negative), and splits by sign when
// lambda > 0.01 and both sides hold more than one node.
//
// Everything a round needs is built on the device (member list by scan,
// induced CSR with original column ids as the reference's NewCol).  The
// whole power iteration is one cooperative kernel: the three reductions per
// iteration (v.k, |y|, |v -+ v0|) are grid-wide barriers instead of the
// reference's four host round trips per iteration.  Reductions are FP64 in
// a fixed order, so a run is deterministic.
#include "pg_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>
#include <string>

namespace cg = cooperative_groups;

namespace {
constexpr int THREADS = 256;
constexpr int MAX_ITER = 10000;
constexpr double EPSILON = 1e-6;
constexpr double LAMBDA = 0.01;

__global__ void k_nm_member(const int32_t* __restrict__ label, int32_t n, int round, int32_t* __restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = label[i] == round;
}

__global__ void k_nm_compact(const int32_t* __restrict__ flag, const long long* __restrict__ off, int32_t n,
                             int32_t* __restrict__ AD)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) AD[off[i]] = i;
}

// In-group degree of every member and the sum of their full degrees.
__global__ void k_nm_subdeg(const int32_t* __restrict__ R, const int32_t* __restrict__ C,
                            const int32_t* __restrict__ flag, const int32_t* __restrict__ AD, int32_t ng,
                            int32_t* __restrict__ kg, unsigned long long* __restrict__ innerM)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = gw; p < ng; p += nw) {
        int i = AD[p];
        int c = 0;
        for (int32_t q = R[i] + lane; q < R[i + 1]; q += 32) c += flag[C[q]];
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) {
            kg[p] = c;
            atomicAdd(innerM, (unsigned long long)(R[i + 1] - R[i]));
        }
    }
}

// Induced CSR (columns keep the original node ids and CSR order).
__global__ void k_nm_subfill(const int32_t* __restrict__ R, const int32_t* __restrict__ C,
                             const int32_t* __restrict__ flag, const int32_t* __restrict__ AD, int32_t ng,
                             const long long* __restrict__ soff, int32_t* __restrict__ sR, int32_t* __restrict__ sC)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int p = gw; p < ng; p += nw) {
        int i = AD[p];
        long long pos = soff[p];
        if (lane == 0) sR[p] = (int32_t)pos;
        if (p == ng - 1 && lane == 0) sR[ng] = (int32_t)soff[ng];
        for (int32_t base = R[i]; base < R[i + 1]; base += 32) {
            int32_t q = base + lane;
            bool in = q < R[i + 1] && flag[C[q]];
            unsigned m = __ballot_sync(0xffffffffu, in);
            if (in) sC[pos + __popc(m & ((1u << lane) - 1u))] = C[q];
            pos += __popc(m);
        }
    }
}

// sumBG (Sub_Partition, Modularity_CPU.cpp:171-173):
//   kg - k * (double)innerM / 2 / M, evaluated in that order.
__global__ void k_nm_sumbg(const int32_t* __restrict__ R, const int32_t* __restrict__ AD,
                           const int32_t* __restrict__ kg, int32_t ng, const unsigned long long* __restrict__ innerM,
                           int M, double* __restrict__ sumBG, double* __restrict__ kdeg)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ng; p += gridDim.x * blockDim.x) {
        int i = AD[p];
        int k = R[i + 1] - R[i];
        double t = __dmul_rn((double)k, (double)*innerM);
        t = __ddiv_rn(t, 2.0);
        t = __ddiv_rn(t, (double)M);
        sumBG[p] = __dsub_rn((double)kg[p], t);
        kdeg[p] = (double)k;
    }
}

struct LVArgs {
    int ng, M;
    const int32_t* AD;
    const int32_t* sR;
    const int32_t* sC;
    const double* kdeg;
    const double* sumBG;
    double beta;
    double* v;
    double* v0;
    double* vv;       // indexed by original node id
    double* part;     // [grid][4]
    double* out;      // lambda, iterations, residual, subP, subN
};

__device__ double block_sum(double x, double* sh)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = x;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sh[q];
    return t;  // valid in thread 0
}

// Fixed-order sum of one column of the per-block partials; every block
// computes the same value.
__device__ double grid_total(const double* part, int col, double* sh_total)
{
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) t += part[b * 4 + col];
        *sh_total = t;
    }
    __syncthreads();
    double t = *sh_total;
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(THREADS) k_nm_lead_vector(LVArgs a)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ double sh[THREADS / 32];
    __shared__ double shv;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int gw = tid >> 5, nw = nthr >> 5;
    const int ng = a.ng;
    for (int p = tid; p < ng; p += nthr) a.v[p] = (double)a.AD[p];
    grid.sync();
    double err1 = 1.0, err2 = 1.0, vnorm = 0.0;
    int iter = 0;
    const double twoM = 2.0;
    while (err1 > EPSILON && err2 > EPSILON && iter < MAX_ITER) {
        // A: v0 = v, scatter to vv, v.k
        double x = 0.0;
        for (int p = tid; p < ng; p += nthr) {
            double vp = a.v[p];
            a.v0[p] = vp;
            a.vv[a.AD[p]] = vp;
            x += vp * a.kdeg[p];
        }
        double bs = block_sum(x, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 0] = bs;
        grid.sync();
        const double v_k = grid_total(a.part, 0, &shv);
        const double c = v_k / twoM / (double)a.M;
        // B: y = A_g v0 - (v.k / 2M) k - (sumBG - beta) v0
        double y2 = 0.0;
        for (int p = gw; p < ng; p += nw) {
            double t = 0.0;
            for (int32_t q = a.sR[p] + lane; q < a.sR[p + 1]; q += 32) t += a.vv[a.sC[q]];
            for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) {
                t -= c * a.kdeg[p] + (a.sumBG[p] - a.beta) * a.v0[p];
                a.v[p] = t;
                y2 += t * t;
            }
        }
        bs = block_sum(y2, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 1] = bs;
        grid.sync();
        vnorm = sqrt(grid_total(a.part, 1, &shv));
        // C: normalise, residuals
        double e1 = 0.0, e2 = 0.0;
        for (int p = tid; p < ng; p += nthr) {
            double vp = a.v[p] / vnorm;
            a.v[p] = vp;
            double d1 = vp - a.v0[p], d2 = vp + a.v0[p];
            e1 += d1 * d1;
            e2 += d2 * d2;
        }
        bs = block_sum(e1, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 2] = bs;
        bs = block_sum(e2, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x * 4 + 3] = bs;
        grid.sync();
        err1 = sqrt(grid_total(a.part, 2, &shv));
        err2 = sqrt(grid_total(a.part, 3, &shv));
        iter++;
        grid.sync();  // partials are rewritten in the next iteration
    }
    // eigenvalue sign from the first entry of largest magnitude
    if (blockIdx.x == 0) {
        __shared__ double bv[THREADS];
        __shared__ int bi[THREADS];
        double best = -1.0;
        int besti = 0x7fffffff;
        long long sp = 0, sn = 0;
        for (int p = threadIdx.x; p < ng; p += blockDim.x) {
            double m = fabs(a.v[p]);
            if (m > best) { best = m; besti = p; }
            sp += a.v[p] > 0.0;
            sn += a.v[p] <= 0.0;
        }
        bv[threadIdx.x] = best;
        bi[threadIdx.x] = besti;
        __shared__ long long csp[THREADS], csn[THREADS];
        csp[threadIdx.x] = sp;
        csn[threadIdx.x] = sn;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = -1.0;
            int ix = 0;
            long long P = 0, Nn = 0;
            for (int t = 0; t < (int)blockDim.x; t++) {
                if (bv[t] > b || (bv[t] == b && bi[t] < ix)) { b = bv[t]; ix = bi[t]; }
                P += csp[t];
                Nn += csn[t];
            }
            double lam = ng > 0 ? ((a.v[ix] * a.v0[ix] > 0) ? vnorm : -vnorm) : 0.0;
            a.out[0] = lam;
            a.out[1] = (double)iter;
            a.out[2] = fmin(err1, err2);
            a.out[3] = (double)P;
            a.out[4] = (double)Nn;
        }
    }
}

__global__ void k_nm_assign(const int32_t* __restrict__ AD, const double* __restrict__ v, int32_t ng, int max_result,
                            double coef, int32_t* __restrict__ label)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < ng; p += gridDim.x * blockDim.x)
        label[AD[p]] = max_result + 1 + (v[p] * coef <= 0.0);
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
    int32_t *label, *flag, *AD, *kg, *sR, *sC;
    long long *off, *soff;
    double *v, *v0, *vv, *sumBG, *kdeg, *part, *out;
    unsigned long long* acc;
    PG_TRY(pg_wst(ctx, "nm.label", (size_t)n + 1, &label));
    PG_TRY(pg_wst(ctx, "nm.flag", (size_t)n + 1, &flag));
    PG_TRY(pg_wst(ctx, "nm.AD", (size_t)n + 1, &AD));
    PG_TRY(pg_wst(ctx, "nm.kg", (size_t)n + 1, &kg));
    PG_TRY(pg_wst(ctx, "nm.off", (size_t)n + 2, &off));
    PG_TRY(pg_wst(ctx, "nm.soff", (size_t)n + 2, &soff));
    PG_TRY(pg_wst(ctx, "nm.sR", (size_t)n + 2, &sR));
    PG_TRY(pg_wst(ctx, "nm.sC", (size_t)nnz + 1, &sC));
    PG_TRY(pg_wst(ctx, "nm.v", (size_t)n + 1, &v));
    PG_TRY(pg_wst(ctx, "nm.v0", (size_t)n + 1, &v0));
    PG_TRY(pg_wst(ctx, "nm.vv", (size_t)n + 1, &vv));
    PG_TRY(pg_wst(ctx, "nm.sumBG", (size_t)n + 1, &sumBG));
    PG_TRY(pg_wst(ctx, "nm.kdeg", (size_t)n + 1, &kdeg));
    PG_TRY(pg_wst(ctx, "nm.acc", (size_t)n + 8, &acc));
    PG_TRY(pg_wst(ctx, "nm.out", 8, &out));
    int per_sm = 0;
    PG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nm_lead_vector, THREADS, 0));
    if (per_sm < 1) return pg_fail(ctx, PG_ERR_INTERNAL, "power iteration kernel cannot be resident");
    const int coop_grid = per_sm * ctx->sm_count;
    PG_TRY(pg_wst(ctx, "nm.part", (size_t)coop_grid * 4 + 4, &part));
    PG_CUDA(ctx, cudaMemsetAsync(label, 0, sizeof(int32_t) * (n + 1), ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(vv, 0, sizeof(double) * (n + 1), ctx->stream));

    const int grid = ctx->sm_count * 4;
    std::vector<int32_t> adjust((size_t)n + 2, 0);
    int Round = 0, Max_Result = 0, Module_Num = 1, Index = 1;
    char line[512];
    if (M == 0) {
        // no edges: the reference's power iteration divides by 2M; the graph
        // is a single module with Q = 0
        std::vector<int32_t> ones(n, 1);
        memcpy(labels, ones.data(), sizeof(int32_t) * n);
        if (Q) *Q = 0.0;
        if (n_modules) *n_modules = 1;
        return PG_OK;
    }
    while (Round <= Max_Result) {
        k_nm_member<<<grid, 256, 0, ctx->stream>>>(label, n, Round, flag);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_scan_counts(ctx, flag, (int64_t*)off, n));
        long long ngl = 0;
        PG_TRY(pg_d2h(ctx, &ngl, off + n, sizeof ngl));
        const int ng = (int)ngl;
        if (ng > 0) {
            k_nm_compact<<<grid, 256, 0, ctx->stream>>>(flag, off, n, AD);
            PG_LAUNCHED(ctx);
            PG_CUDA(ctx, cudaMemsetAsync(acc, 0, sizeof(unsigned long long), ctx->stream));
            k_nm_subdeg<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, flag, AD, ng, kg, acc);
            PG_LAUNCHED(ctx);
            PG_TRY(pg_scan_counts(ctx, kg, (int64_t*)soff, ng));
            k_nm_subfill<<<grid, 256, 0, ctx->stream>>>(g->R, g->C, flag, AD, ng, soff, sR, sC);
            PG_LAUNCHED(ctx);
            k_nm_sumbg<<<grid, 256, 0, ctx->stream>>>(g->R, AD, kg, ng, acc, M, sumBG, kdeg);
            PG_LAUNCHED(ctx);
            double res[2][5];
            LVArgs a = {ng, M, AD, sR, sC, kdeg, sumBG, 0.0, v, v0, vv, part, out};
            for (int pass = 0; pass < 2; pass++) {
                void* args[] = {(void*)&a};
                PG_CUDA(ctx, cudaLaunchCooperativeKernel((void*)k_nm_lead_vector, dim3(coop_grid), dim3(THREADS),
                                                         args, 0, ctx->stream));
                PG_LAUNCHED(ctx);
                PG_TRY(pg_d2h(ctx, res[pass], out, sizeof(double) * 5));
                if (pass == 0) {
                    // shift rule: CPU variant lambda < 0 (Modularity_CPU.cpp:177),
                    // GPU variant lambda < -LAMBDA for large groups (modularity_GPU.cu:374)
                    const double below = ng > gpu_rule_above ? -LAMBDA : 0.0;
                    if (!(res[0][0] < below)) break;
                    a.beta = -res[0][0];
                }
            }
            const bool shifted = a.beta != 0.0;
            const double lambda = shifted ? res[0][0] + res[1][0] : res[0][0];
            const double* fin = shifted ? res[1] : res[0];
            const long long subP = (long long)fin[3], subN = (long long)fin[4];
            const bool issub = lambda > LAMBDA && subP > 1 && subN > 1;
            if (log) {
                int len = snprintf(line, sizeof line, "Round:\t%d\tnumber of nodes:\t%d\tIterations:\t%d\tresidual:\t%g\t",
                                   Round, ng, (int)res[0][1], res[0][2]);
                if (shifted)
                    len += snprintf(line + len, sizeof line - len, "Iterations:\t%d\tresidual:\t%g\t", (int)res[1][1],
                                    res[1][2]);
                snprintf(line + len, sizeof line - len, "Eigen Value: %g\tDivide?: %d", lambda, (int)issub);
                log(line, user);
            }
            if (issub) {
                k_nm_assign<<<grid, 256, 0, ctx->stream>>>(AD, v, ng, Max_Result, (double)(subP - subN) + 0.5, label);
                PG_LAUNCHED(ctx);
                Max_Result += 2;
            } else {
                if (Round >= (int)adjust.size()) adjust.resize(Round + 1, 0);
                adjust[Round] = Index++;
            }
            Module_Num += issub;
        }
        Round++;
    }
    // Q from module degree sums (Modularity_CPU.cpp:116-124 in closed form)
    unsigned long long* Kc = acc + 2;
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
    std::vector<int32_t> raw(n);
    PG_TRY(pg_d2h(ctx, raw.data(), label, sizeof(int32_t) * n));
    for (int i = 0; i < n; i++) labels[i] = adjust[raw[i]];
    if (Q) *Q = q;
    if (n_modules) *n_modules = Module_Num;
    if (log) {
        snprintf(line, sizeof line, "Number of Modules: %d,\tQ=%.6g", Module_Num, q);
        log(line, user);
    }
    return PG_OK;
}
