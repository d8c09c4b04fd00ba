// runner.cu -- a cohort of subjects through the whole path in one call: the
// chain of reference tools CUCorMat -> Degree -> Cp -> BFS_MulCPU / CUBC ->
// Newman_Modularity -> Maslov -> Cp / BFS_MulCPU on the surrogates ->
// SmallWorldProperty, which the reference runs as separate programs over a
// directory of files, here one device-resident pass per subject (the graph
// never leaves HBM).
//
// The surrogates dominate a cohort run (config: 20 per subject, each a
// Maslov rewiring of 10 x |E| attempts plus clustering and all-source hop
// paths).  Their chain -- rewiring (one cooperative launch for all rounds),
// the surrogate's rows (R is the subject's: degrees are preserved),
// clustering, hop paths (one cooperative launch for all batches and levels)
// and a collect kernel that files the surrogate's Cp mean and Lp under the
// replay index -- enqueues no host round trip and allocates nothing once
// sized.  Surrogate 0 runs directly (it sizes the workspace, sets kernel
// attributes and runs the autotuner on the real surrogate); the chain is then
// captured into a CUDA graph once per subject and replayed for the other
// surrogates, the replay index selecting the seed from a device array.
#include "pg_internal.cuh"
#include "clustering.cuh"
#include "maslov.cuh"
#include "paths.cuh"
#include <cstring>
#include <vector>

namespace {
// seed of surrogate r of subject s: distinct for every (s, r)
uint64_t surrogate_seed(uint64_t base, int32_t s, int32_t r)
{
    uint64_t z = base + 0x9E3779B97F4A7C15ULL * (uint64_t)(s + 1) + (uint64_t)r;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct GraphGuard {
    pg_graph* g = nullptr;
    ~GraphGuard() { pg_graph_free(g); }
};

struct ExecGuard {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~ExecGuard()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// Files the surrogate's results under the replay index and advances it.
__global__ void k_sr_collect(const double* __restrict__ cp_mean, const double* __restrict__ path_out,
                             double* __restrict__ cp_r, double* __restrict__ lp_r, int* __restrict__ round)
{
    const int r = *round;
    cp_r[r] = *cp_mean;
    lp_r[r] = path_out[1];
    *round = r + 1;
}

struct SurrogateChain {
    pg_graph sg;              // the surrogate: R shared with the subject graph, C/V in the workspace
    MsArgs ms;
    BinaryCpArgs bin;
    OnnelaArgs onn;
    PathArgs pa;
    bool weighted;
    float* cp;
    double* cp_mean;
    double *cp_r, *lp_r;
    int* round;
};

pg_status chain_enqueue(pg_ctx* ctx, const pg_graph* g, SurrogateChain& c)
{
    PG_TRY(ms_enqueue(ctx, g, &c.ms));
    PG_TRY(ms_rows_enqueue(ctx, g, &c.ms, c.sg.C, c.sg.V));
    if (c.weighted) PG_TRY(onnela_enqueue(ctx, &c.onn));
    else PG_TRY(binary_cp_enqueue(ctx, &c.bin, c.sg.R, c.sg.C, c.sg.n, c.cp, nullptr, c.cp_mean));
    PG_TRY(paths_enqueue(ctx, &c.pa));
    k_sr_collect<<<1, 1, 0, ctx->stream>>>(c.cp_mean, c.pa.out, c.cp_r, c.lp_r, c.round);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

// Clustering means and Lp of n_random surrogates of g into cp_r / lp_r (host).
pg_status run_surrogates(pg_ctx* ctx, const pg_graph* g, int32_t subject, const pg_run_opts& o, double* cp_r,
                         double* lp_r, int32_t* replays)
{
    const int nr = o.n_random;
    SurrogateChain c{};
    c.weighted = g->V != nullptr;
    c.sg.ctx = ctx;
    c.sg.device = ctx->device;
    c.sg.n = g->n;
    c.sg.nnz = g->nnz;
    c.sg.R = g->R;
    PG_TRY(pg_wst(ctx, "sr.C", (size_t)g->nnz + 1, &c.sg.C));
    if (c.weighted) PG_TRY(pg_wst(ctx, "sr.V", (size_t)g->nnz + 1, &c.sg.V));
    PG_TRY(pg_wst(ctx, "sr.cp", (size_t)g->n + 1, &c.cp));
    PG_TRY(pg_wst(ctx, "sr.cpmean", 1, &c.cp_mean));
    PG_TRY(pg_wst(ctx, "sr.cp_r", (size_t)nr, &c.cp_r));
    PG_TRY(pg_wst(ctx, "sr.lp_r", (size_t)nr, &c.lp_r));
    PG_TRY(pg_wst(ctx, "sr.round", 1, &c.round));
    uint64_t* seeds;
    PG_TRY(pg_wst(ctx, "sr.seeds", (size_t)nr, &seeds));
    std::vector<uint64_t> hs((size_t)nr);
    for (int r = 0; r < nr; r++) hs[r] = surrogate_seed(o.seed, subject, r);
    PG_TRY(pg_h2d(ctx, seeds, hs.data(), sizeof(uint64_t) * nr));
    PG_CUDA(ctx, cudaMemsetAsync(c.round, 0, sizeof(int), ctx->stream));
    const int64_t attempts = o.swaps_per_edge * (g->nnz / 2);
    PG_TRY(ms_prepare(ctx, g, 0, attempts, &c.ms));
    c.ms.seed_dev = seeds;
    c.ms.round_dev = c.round;
    // surrogate 0, directly: its rows must exist before the clustering and
    // path set-up look at them (the autotuner runs on this surrogate)
    PG_TRY(ms_enqueue(ctx, g, &c.ms));
    PG_TRY(ms_rows_enqueue(ctx, g, &c.ms, c.sg.C, c.sg.V));
    if (c.weighted) {
        const pg_graph* one[1] = {&c.sg};
        PG_TRY(onnela_prepare(ctx, one, 1, 0, c.cp, c.cp_mean, &c.onn));
        PG_TRY(onnela_enqueue(ctx, &c.onn));
    } else {
        PG_TRY(binary_cp_prepare(ctx, g->n, &c.bin));
        PG_TRY(binary_cp_enqueue(ctx, &c.bin, c.sg.R, c.sg.C, c.sg.n, c.cp, nullptr, c.cp_mean));
    }
    PG_TRY(paths_prepare(ctx, &c.sg, 0, &c.pa));
    PG_TRY(paths_enqueue(ctx, &c.pa));
    k_sr_collect<<<1, 1, 0, ctx->stream>>>(c.cp_mean, c.pa.out, c.cp_r, c.lp_r, c.round);
    PG_LAUNCHED(ctx);
    // surrogates 1.., as replays of one captured chain
    int done = 1;
    *replays = 0;
    if (nr > 1 && o.cuda_graphs) {
        ExecGuard eg;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        pg_status st = e == cudaSuccess ? chain_enqueue(ctx, g, c) : PG_ERR_CUDA;
        if (e == cudaSuccess) {
            cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &eg.graph);
            if (st == PG_OK && e2 == cudaSuccess)
                e2 = cudaGraphInstantiate(&eg.exec, eg.graph, 0);
            if (st == PG_OK && e2 != cudaSuccess) st = PG_ERR_CUDA;
        }
        if (st == PG_OK) {
            for (; done < nr; done++) PG_CUDA(ctx, cudaGraphLaunch(eg.exec, ctx->stream));
            *replays = nr - 1;
        } else {
            (void)cudaGetLastError();   // capture not available: enqueue the chain directly below
            ctx->err.clear();
        }
    }
    for (; done < nr; done++) PG_TRY(chain_enqueue(ctx, g, c));
    PG_TRY(pg_d2h(ctx, cp_r, c.cp_r, sizeof(double) * nr));
    PG_TRY(pg_d2h(ctx, lp_r, c.lp_r, sizeof(double) * nr));
    return PG_OK;
}

pg_status run_one(pg_ctx* ctx, pg_subject& sj, int32_t index, const pg_run_opts& o)
{
    if (!sj.bold || sj.N < 1 || sj.T < 1)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_run_subjects: subject %d has no series (N=%d T=%d)", index, sj.N,
                       sj.T);
    GraphGuard gg;
    pg_build_info info;
    PG_TRY(pg_build_graph(ctx, sj.bold, sj.N, sj.T, &o.build, &gg.g, &info));
    const pg_graph* g = gg.g;
    sj.edges = info.edges;
    sj.tau = info.tau;
    const bool weighted = o.build.weighted != 0;
    if (sj.degree) {
        int32_t iso = 0;
        PG_TRY(pg_degree(ctx, g, sj.degree, &iso));
    }
    const bool want_sw = o.n_random > 0;
    sj.cp_mean = 0.0;
    if (sj.cp || want_sw) {
        std::vector<float> tmp;
        float* cp = sj.cp;
        if (!cp) {
            tmp.resize((size_t)sj.N);
            cp = tmp.data();
        }
        PG_TRY(pg_clustering(ctx, g, weighted ? 1 : 0, 0, cp, nullptr, &sj.cp_mean));
    }
    sj.lp = 0.0;
    if (sj.bc) {
        PG_TRY(pg_betweenness(ctx, g, sj.bc, nullptr, sj.eff, &sj.lp));
    } else if (sj.eff || want_sw) {
        PG_TRY(pg_paths(ctx, g, sj.eff, nullptr, &sj.lp, nullptr, 0, nullptr));
    }
    sj.Q = 0.0;
    sj.n_modules = 0;
    if (sj.modules) {
        if (weighted) PG_TRY(pg_newman_weighted(ctx, g, nullptr, 25000, sj.modules, &sj.Q, &sj.n_modules, nullptr,
                                                nullptr));
        else PG_TRY(pg_newman(ctx, g, 25000, sj.modules, &sj.Q, &sj.n_modules, nullptr, nullptr));
    }
    sj.gamma = sj.lambda = sj.sigma = 0.0;
    sj.surrogate_graph_replays = 0;
    if (want_sw) {
        std::vector<double> cp_r((size_t)o.n_random), lp_r((size_t)o.n_random);
        PG_TRY(run_surrogates(ctx, g, index, o, cp_r.data(), lp_r.data(), &sj.surrogate_graph_replays));
        PG_TRY(pg_smallworld(sj.cp_mean, cp_r.data(), o.n_random, sj.lp, lp_r.data(), o.n_random, &sj.gamma,
                             &sj.lambda, &sj.sigma));
    }
    return PG_OK;
}
}  // namespace

extern "C" void pg_run_opts_default(pg_run_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof *o);
    pg_build_opts_default(&o->build);
    o->n_random = 0;
    o->swaps_per_edge = 2;
    o->seed = 1;
    o->cuda_graphs = 1;
}

extern "C" uint64_t pg_surrogate_seed(uint64_t base, int32_t subject, int32_t r)
{
    return surrogate_seed(base, subject, r);
}

extern "C" pg_status pg_run_subjects(pg_ctx* ctx, pg_subject* subjects, int32_t n, const pg_run_opts* opts)
{
    if (!ctx || (n > 0 && !subjects) || n < 0) return pg_fail(ctx, PG_ERR_INVALID, "pg_run_subjects: bad arguments");
    pg_run_opts o;
    if (opts) o = *opts;
    else pg_run_opts_default(&o);
    if (o.n_random < 0 || o.swaps_per_edge < 0)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_run_subjects: negative surrogate count or swaps");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    for (int32_t s = 0; s < n; s++) PG_TRY(run_one(ctx, subjects[s], s, o));
    return PG_OK;
}
