// runner.cu -- a cohort of subjects through the whole path in one call: the
// chain of reference tools CUCorMat -> Degree -> Cp -> BFS_MulCPU / CUBC ->
// Newman_Modularity -> Maslov -> SmallWorldProperty, which the reference runs
// as separate programs over a directory of files, here one device-resident
// pass per subject (the graph never leaves HBM).  Host code over the other
// entry points; no kernels of its own.
#include "pg_internal.cuh"
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
    const int32_t kind = o.build.weighted ? 1 : 0;   // Onnela for weighted graphs
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
        PG_TRY(pg_clustering(ctx, g, kind, 0, cp, nullptr, &sj.cp_mean));
    }
    sj.lp = 0.0;
    if (sj.bc) {
        PG_TRY(pg_betweenness(ctx, g, sj.bc, nullptr, sj.eff, &sj.lp));
    } else if (sj.eff || want_sw) {
        PG_TRY(pg_paths(ctx, g, sj.eff, nullptr, &sj.lp, nullptr, 0, nullptr));
    }
    sj.Q = 0.0;
    sj.n_modules = 0;
    if (sj.modules) PG_TRY(pg_newman(ctx, g, 25000, sj.modules, &sj.Q, &sj.n_modules, nullptr, nullptr));
    sj.gamma = sj.lambda = sj.sigma = 0.0;
    if (want_sw) {
        std::vector<double> cp_r((size_t)o.n_random), lp_r((size_t)o.n_random);
        const int64_t attempts = o.swaps_per_edge * (g->nnz / 2);
        for (int32_t r = 0; r < o.n_random; r++) {
            GraphGuard rg;
            PG_TRY(pg_maslov(ctx, g, surrogate_seed(o.seed, index, r), attempts, &rg.g, nullptr));
            std::vector<float> cpr((size_t)sj.N);
            PG_TRY(pg_clustering(ctx, rg.g, kind, 0, cpr.data(), nullptr, &cp_r[r]));
            PG_TRY(pg_paths(ctx, rg.g, nullptr, nullptr, &lp_r[r], nullptr, 0, nullptr));
        }
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
    for (int32_t s = 0; s < n; s++) PG_TRY(run_one(ctx, subjects[s], s, o));
    return PG_OK;
}
