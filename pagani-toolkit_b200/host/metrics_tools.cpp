// metrics_tools.cpp -- the reference's per-metric console tools over the
// C ABI.  One binary per tool is built from this file (PG_TOOL_<NAME>); argv,
// directory scanning and output names follow the reference:
//   Degree <dir>                              U/Degree/Degree/Degree.cpp (W: strength)
//   Cp <dir> <n_rand> [1|2] <g|n|k|gn|gk|nk|gnk>   U/Cp/Cp/Cp_main.cpp, W/Cp/Cp/Cp_main.cpp
//   BFS_MulCPU <dir> <n_rand> <n|g|b>         U/BFS_MulCPU/BFS_MulCPU/MUBFS_LP_main.cpp
//   CUBFW_Lp <dir> <n_rand> <g|n|l|gn|gl|nl|gnl>  W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp_main.cpp
//   CUBC <dir>                                U/BC/CUBC/CUBC_main.cpp
//   Newman_Modularity <dir> <n_rand>          U/cuda_EC/cuda_EC/modularity_GPU.cu:532-717
//   Newman_Modularity_weighted <dir> <n_rand> W/Newman_Modularity_GPU/CUmodularity/modularity_GPU.cu:527-724
//   CUEC <dir>                                U/CUEC/CUEC/CUEC_unweighted.cu:216-312, W/CUEC/weighted-net.cu:220-331
//   PC_CPU <dir>                              W/PC_CPU/PC_CPU/main.cpp:8-205
//   Maslov <file.csr>                         W/Maslov/Maslov/Maslov_main.cpp
//   SmallWorldProperty <dir>                  W/SmallWorldProperty/SmallWorldProperty.cpp
// Random surrogates use pg_maslov with 2*M attempts (the reference's
// Rewire count, Maslov.cpp:19) and a seed from PAGANI_SEED.
#include <dirent.h>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "formats.h"

using pgio::Csr;

[[maybe_unused]] static std::vector<std::string> csr_files(const char* dir)
{
    std::vector<std::string> f = pgio::list_dir(dir, ".csr");
    printf("%zu files to be processed.\n", f.size());
    return f;
}

[[maybe_unused]] static bool load(const std::string& path, Csr& g)
{
    std::string err;
    if (!pgio::read_csr(path, g, err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return false;
    }
    return true;
}

[[maybe_unused]] static pg_graph* surrogate(pg_ctx* ctx, pg_graph* g, uint64_t salt)
{
    int64_t nnz = 0;
    pg_graph_info(g, nullptr, &nnz, nullptr);
    pg_graph* r = nullptr;
    int64_t committed = 0;
    pgio::check(ctx, pg_maslov(ctx, g, pgio::surrogate_seed(salt), nnz /* 2*M attempts */, &r, &committed), "pg_maslov");
    return r;
}

// flag parsing of the g/n/k style argument (Cp_main.cpp:75-97)
[[maybe_unused]] static void flags(const char* s, const char* letters, bool* out)
{
    for (int q = 0; letters[q]; q++) out[q] = strchr(s, letters[q]) != nullptr;
}

#if defined(PG_TOOL_DEGREE)
int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "Input format: Degree dir_for_csr\n"); return 1; }
    pg_ctx* ctx = pgio::open_ctx();
    FILE* iso_file = fopen(pgio::join(argv[1], "isolated_v_mark.txt").c_str(), "w");
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> deg(c.n());
        int32_t iso = 0;
        pgio::check(ctx, pg_degree(ctx, g, deg.data(), &iso), "pg_degree");
        if (iso_file) fprintf(iso_file, "%d\n", iso);
        pgio::write_nm(pgio::stem(path) + "_deg.nm", deg);
        pg_graph_free(g);
    }
    if (iso_file) fclose(iso_file);
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_CP)
int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "Input format: Cp dir_for_csr num_of_random_networks [1|2] parameter_type\n"); return 1; }
    const int nrand = atoi(argv[2]);
    int kind_arg = 2;                      // weighted: 2 = Onnela (default), 1 = Barrat
    const char* type = argv[3];
    if (argc >= 5) { kind_arg = atoi(argv[3]); type = argv[4]; }
    bool f[3];
    flags(type, "gnk", f);
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
        const bool weighted = !c.V.empty();
        if (weighted && kind_arg == 1) { fprintf(stderr, "Barrat clustering is not provided by this build\n"); return 1; }
        const int kind = weighted ? 1 : 0;
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> cp(c.n());
        double mean = 0;
        pgio::check(ctx, pg_clustering(ctx, g, kind, 0, cp.data(), nullptr, &mean), "pg_clustering");
        printf("average Cp:\t%.6g\n", mean);
        if (f[1]) pgio::write_nm(pgio::stem(path) + "_cp.nm", cp);
        std::vector<double> means = {mean};
        double rsum = 0;
        for (int l = 0; l < nrand; l++) {
            pg_graph* r = surrogate(ctx, g, (uint64_t)l);
            double m = 0;
            pgio::check(ctx, pg_clustering(ctx, r, kind, 0, cp.data(), nullptr, &m), "pg_clustering");
            means.push_back(m);
            rsum += m;
            pg_graph_free(r);
        }
        if (f[0]) pgio::write_values(pgio::stem(path) + "_cp.txt", means);
        if (f[2]) pgio::write_values(pgio::stem(path) + "_gamma.txt", {mean / (rsum / nrand)});
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_BFS)
int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "Input format: BFS_MulCPU dir_for_csr num_of_random_networks n|g|b\n"); return 1; }
    const int nrand = atoi(argv[2]);
    const char t = argv[3][0];
    const bool nodal = t == 'n' || t == 'b', global = t == 'g' || t == 'b';
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> eff(c.n());
        double lp = 0;
        pgio::check(ctx, pg_paths(ctx, g, eff.data(), nullptr, &lp, nullptr, 0, nullptr), "pg_paths");
        if (nodal) pgio::write_nm(pgio::stem(path) + "_eff.nm", eff);
        if (global) {
            printf("average Lp:\t%.6g\n", lp);
            std::vector<double> lps = {lp};
            for (int l = 0; l < nrand; l++) {
                pg_graph* r = surrogate(ctx, g, (uint64_t)l);
                double x = 0;
                pgio::check(ctx, pg_paths(ctx, r, nullptr, nullptr, &x, nullptr, 0, nullptr), "pg_paths");
                lps.push_back(x);
                pg_graph_free(r);
            }
            pgio::write_values(pgio::stem(path) + "_Lp.txt", lps);
        }
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_BFW)
int main(int argc, char** argv)
{
    if (argc < 3) { fprintf(stderr, "Input format: CUBFW_Lp dir_for_csr num_of_random_networks parameter_type\n"); return 1; }
    const int nrand = argc >= 4 ? atoi(argv[2]) : 0;
    bool f[3] = {true, true, true};
    if (argc >= 4) flags(argv[3], "gnl", f);
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> eff(c.n());
        double lp = 0;
        pgio::check(ctx, pg_fw_paths(ctx, g, nullptr, eff.data(), &lp), "pg_fw_paths");
        if (f[1]) pgio::write_nm(pgio::stem(path) + "_eff.nm", eff);
        printf("average Lp:\t%.6g\n", lp);
        std::vector<double> lps = {lp};
        double rsum = 0;
        for (int l = 0; l < nrand; l++) {
            pg_graph* r = surrogate(ctx, g, (uint64_t)l);
            double x = 0;
            pgio::check(ctx, pg_fw_paths(ctx, r, nullptr, eff.data(), &x), "pg_fw_paths");
            lps.push_back(x);
            rsum += x;
            pg_graph_free(r);
        }
        if (f[0]) pgio::write_values(pgio::stem(path) + "_Lp.txt", lps);
        if (f[2]) pgio::write_values(pgio::stem(path) + "_lambda.txt", {lp / (rsum / nrand)});
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_BC)
int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "Input format: CUBC dir_for_csr\n"); return 1; }
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> bc(c.n());
        pgio::check(ctx, pg_betweenness(ctx, g, bc.data(), nullptr, nullptr, nullptr), "pg_betweenness");
        pgio::write_nm(pgio::stem(path) + "_bc.nm", bc);
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_NEWMAN)
// The unweighted tool writes int32 labels to X.modu; the weighted build
// (PG_WEIGHTED_TOOL) uses the file's values and writes float labels to
// X_modu.nm, and partitions its random surrogates with the original values
// (modularity_GPU.cu of the weighted package, :655-662 and :114-123).
static void log_line(const char* line, void* user) { fprintf((FILE*)user, "%s\n", line); }
int main(int argc, char** argv)
{
#ifdef PG_WEIGHTED_TOOL
    const char* name = "Newman_Modularity_weighted";
#else
    const char* name = "Newman_Modularity";
#endif
    if (argc != 3) { fprintf(stderr, "Input format: %s dir_for_csr num_of_random_networks\n", name); return 1; }
    const int nrand = atoi(argv[2]);
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        Csr c;
        if (!load(path, c)) continue;
#ifdef PG_WEIGHTED_TOOL
        if (c.V.empty()) {
            fprintf(stderr, "Your csr file %s has no weights\n", path.c_str());
            continue;
        }
#endif
        pg_graph* g = pgio::upload(ctx, c);
        FILE* log = fopen((pgio::stem(path) + "_modu.txt").c_str(), "w");
        std::vector<int32_t> labels(c.n());
        double Q = 0;
        int32_t nm = 0;
#ifdef PG_WEIGHTED_TOOL
        pgio::check(ctx, pg_newman_weighted(ctx, g, g, 25000, labels.data(), &Q, &nm, log ? log_line : nullptr, log),
                    "pg_newman_weighted");
        printf("Number of Modules: %d,\tQ=%.6g\n", nm, Q);
        pgio::write_nm(pgio::stem(path) + "_modu.nm", std::vector<float>(labels.begin(), labels.end()));
#else
        pgio::check(ctx, pg_newman(ctx, g, 25000, labels.data(), &Q, &nm, log ? log_line : nullptr, log), "pg_newman");
        printf("Number of Modules: %d,\tQ=%.6g\n", nm, Q);
        pgio::write_modu(pgio::stem(path) + ".modu", labels);
#endif
        for (int l = 0; l < nrand; l++) {   // the reference logs the random partitions only
            pg_graph* r = surrogate(ctx, g, (uint64_t)l);
#ifdef PG_WEIGHTED_TOOL
            pgio::check(ctx, pg_newman_weighted(ctx, r, g, 25000, labels.data(), &Q, &nm, log ? log_line : nullptr, log),
                        "pg_newman_weighted");
#else
            pgio::check(ctx, pg_newman(ctx, r, 25000, labels.data(), &Q, &nm, log ? log_line : nullptr, log), "pg_newman");
#endif
            pg_graph_free(r);
        }
        if (log) fclose(log);
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_EC)
// Eigenvector centrality of every .csr in the directory: <stem>_ec.nm and
// <stem>_evalue.txt.  A file with weights is treated as the weighted tool
// does (weights used, y = A x of the last step written); a binary file as
// the unweighted tool does (the normalised vector written).
int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "Input format: CUEC dir_for_csr\n"); return 1; }
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& fn : csr_files(argv[1])) {
        std::string path = pgio::join(argv[1], fn);
        printf("\ncalculating eigenvalue centrality for %s ...\n", path.c_str());
        Csr c;
        if (!load(path, c)) continue;
        const bool weighted = !c.V.empty();
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<double> ec(c.n());
        double lam = 0.0, res = 0.0;
        int32_t it = 0;
        pgio::check(ctx, pg_eigen_centrality(ctx, g, weighted ? 1 : 0, ec.data(), &lam, &it, &res),
                    "pg_eigen_centrality");
        printf("Iterations:\t%d\tresidual:\t%g\teigenvalue:\t%g\t\n", it, res, lam);
        std::vector<float> ecf(ec.begin(), ec.end());
        pgio::write_nm(pgio::stem(path) + "_ec.nm", ecf);
        // the unweighted tool returns the eigenvalue as float before printing it
        pgio::write_values(pgio::stem(path) + "_evalue.txt", {weighted ? lam : (double)(float)lam});
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_PC)
// Participation coefficient of every X.csr in the directory (names holding
// ".csr"; the first ".csr" is cut to form X) whose module file X_modu.nm
// (float labels) exists: X_pc.nm and X_pc.nm_Normalized.nm.
int main(int argc, char** argv)
{
    if (argc != 2 && argc != 3) {
        fprintf(stderr, "No Directory Input\nInput format: PC_CPU dir_for_csr_and_modu\n");
        return 1;
    }
    std::vector<std::string> names;
    if (DIR* dp = opendir(argv[1])) {
        while (dirent* e = readdir(dp)) {
            std::string nm = e->d_name;
            const size_t pos = nm.find(".csr");
            if (pos != std::string::npos) names.push_back(nm.replace(pos, 4, ""));
        }
        closedir(dp);
    } else {
        printf("can't open %s\n", argv[1]);
        return 1;
    }
    std::sort(names.begin(), names.end());
    pg_ctx* ctx = pgio::open_ctx();
    for (const std::string& x : names) {
        const std::string base = pgio::join(argv[1], x);
        printf("calculate participant coefficient of %s.csr\n\n", base.c_str());
        Csr c;
        if (!load(base + ".csr", c)) continue;
        std::vector<float> mod;
        if (!pgio::read_nm(base + "_modu.nm", mod) || (int)mod.size() != c.n()) {
            printf("%s_modu.nm not found!\n", base.c_str());
            continue;
        }
        pg_graph* g = pgio::upload(ctx, c);
        std::vector<float> pc(c.n()), pn(c.n());
        int32_t K = 0;
        pgio::check(ctx, pg_participation(ctx, g, mod.data(), pc.data(), pn.data(), &K), "pg_participation");
        pgio::write_nm(base + "_pc.nm", pc);
        pgio::write_nm(base + "_pc.nm_Normalized.nm", pn);
        pg_graph_free(g);
    }
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_MASLOV)
int main(int argc, char** argv)
{
    if (argc != 2) { fprintf(stderr, "Input format example: Maslov data_avr_20_0.06.csr\n"); return 1; }
    std::string path = argv[1];
    Csr c;
    if (!load(path, c)) return 1;
    pg_ctx* ctx = pgio::open_ctx();
    pg_graph* g = pgio::upload(ctx, c);
    pg_graph* r = surrogate(ctx, g, 0);
    Csr out = pgio::download(ctx, r);
    std::string dst = path.size() > 4 ? path.substr(0, path.size() - 4) + "_Maslov.csr" : path + "_Maslov.csr";
    if (!pgio::write_csr(dst, out)) fprintf(stderr, "cannot write %s\n", dst.c_str());
    pg_graph_free(r);
    pg_graph_free(g);
    pg_destroy(ctx);
    return 0;
}
#elif defined(PG_TOOL_SMALLWORLD)
// Pairs *_lambda.txt with *_gamma.txt whose names agree in characters 1-4 and
// in the 5 characters after "spa" (SmallWorldProperty.cpp:104-126); writes
// sigma = gamma / lambda to <lambda name up to its last '_'>_smallWorld.txt.
static std::string feat(const std::string& n, int which)
{
    if (which == 0) return n.size() > 5 ? n.substr(1, 4) : n;
    size_t p = n.find("spa");
    return p == std::string::npos ? "" : n.substr(p + 3, 5);
}
int main(int argc, char** argv)
{
    if (argc < 2) { fprintf(stderr, "Input format: SmallWorldProperty dir\n"); return 1; }
    std::vector<std::string> all = pgio::list_dir(argv[1], ".txt"), lam, gam;
    for (const std::string& n : all) {
        if (n.size() > 11 && n.substr(n.size() - 11) == "_lambda.txt") lam.push_back(n);
        if (n.size() > 10 && n.substr(n.size() - 10) == "_gamma.txt") gam.push_back(n);
    }
    if (lam.empty()) fprintf(stderr, "Lack lambda files.\n");
    if (gam.empty()) fprintf(stderr, "Lack gamma files.\n");
    std::vector<bool> used(gam.size(), false);
    for (const std::string& l : lam) {
        for (size_t j = 0; j < gam.size(); j++) {
            if (used[j] || feat(l, 0) != feat(gam[j], 0) || feat(l, 1) != feat(gam[j], 1)) continue;
            used[j] = true;
            double lambda = 0, gamma = 0;
            if (!pgio::read_first_value(pgio::join(argv[1], l), lambda) ||
                !pgio::read_first_value(pgio::join(argv[1], gam[j]), gamma))
                break;
            double g = 0, lm = 0, sigma = 0;
            pg_smallworld(gamma, &g, 0, lambda, &lm, 0, nullptr, nullptr, nullptr);
            sigma = gamma / lambda;
            std::string base = l.substr(0, l.find_last_of('_'));
            printf("Small world property equals %.6g\n", sigma);
            pgio::write_values(pgio::join(argv[1], base + "_smallWorld.txt"), {sigma});
            break;
        }
    }
    return 0;
}
#else
#error "build with -DPG_TOOL_<NAME>"
#endif
