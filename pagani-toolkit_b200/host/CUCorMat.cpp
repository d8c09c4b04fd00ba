// CUCorMat -- network construction, same argv and outputs as the reference
// tool (U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:51-378; weighted twin
// W/CorMat/CUCorMat/CUCorMat/CorMat.cpp, selected here by building this file
// with -DPG_WEIGHTED_TOOL).
//
//   CUCorMat <dir> [<mask.nii>] <mask_thr> <n|yf|yn|bf|bn> <y|n save .cormat> <r|s> <thr...>
//
// Every *.nii in <dir> except mask.nii is a subject; the mask is <dir>/mask.nii
// (source version) or the path given after <dir> (manual's form).  Voxels
// with mask >= mask_thr are kept.  For each threshold the graph is written
// as <stem>_<N>_spa%.3f%%_cor%.3f.csr (weighted: ..._weighted.csr, CSR + r).
// to_average (CorMat.cpp:187-189, :380-620): n = one graph per subject,
// y = one graph of the subject average, b = both; the second letter picks
// the plain (n) or Fisher-z (f) average.  The averaged outputs are
// <dir>/<dir name>_<subjects>_<N>[.cormat | _spa%.3f%%_cor%.3f.csr] (no
// _weighted suffix, and no 1e-6 shift of the r threshold, in either tool:
// W CorMat.cpp:521-600).  Unlike the reference, an average mode other than
// these five is an error (the reference leaves the sum at zero).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "formats.h"

#ifdef PG_WEIGHTED_TOOL
static const bool kWeighted = true;
#else
static const bool kWeighted = false;
#endif

// Base name of the averaged outputs (CorMat.cpp:136-137, :521-527): one
// trailing separator is dropped, then <dir>/<last component>, or <dir>/ when
// the path has no separator, followed by _<subjects>_<N>.
static std::string cohort_base(std::string dir, size_t subjects, int N)
{
    if (dir.size() > 1 && dir.back() == '/') dir.pop_back();
    const size_t s = dir.find_last_of('/');
    const std::string base = s == std::string::npos ? dir + "/" : dir + dir.substr(s);
    return base + "_" + std::to_string(subjects) + "_" + std::to_string(N);
}

static bool is_file(const std::string& p)
{
    FILE* f = fopen(p.c_str(), "rb");
    if (!f) return false;
    fclose(f);
    return true;
}

int main(int argc, char** argv)
{
    if (argc < 7) {
        fprintf(stderr,
                "Input format: CUCorMat Dir_for_BOLD [mask.nii] threshold_for_mask(0~1) to_average(yf/yn/bf/bn/n) "
                "to_save_cormatrix(y/n) threshold_type(r/s) threshold(s)\n"
                "For example: CUCorMat /data/BOLD 0.5 n n r 0.2 0.25 0.3\n");
        return 1;
    }
    std::string dir = argv[1];
    int a = 2;
    std::string mask_path = pgio::join(dir, "mask.nii");
    if (std::string(argv[2]).size() > 4 && std::string(argv[2]).substr(std::string(argv[2]).size() - 4) == ".nii" &&
        is_file(argv[2])) {
        mask_path = argv[2];
        a = 3;
    }
    if (argc < a + 5) {
        fprintf(stderr, "missing arguments\n");
        return 1;
    }
    const float prob_cut = (float)atof(argv[a]);
    const char avg = (char)tolower(argv[a + 1][0]);
    const char save = argv[a + 2][0];
    const char mode = argv[a + 3][0];
    const bool per_subject = avg == 'n' || avg == 'b';
    const bool average = avg == 'y' || avg == 'b';
    const char avg_kind = average ? (char)tolower(argv[a + 1][1]) : 0;
    if ((!per_subject && !average) || (average && avg_kind != 'f' && avg_kind != 'n')) {
        fprintf(stderr, "to_average must be n, yf, yn, bf or bn (got %s)\n", argv[a + 1]);
        return 1;
    }
    const bool rmode = (mode == 'r' || mode == 'R');
    if (!rmode && mode != 's' && mode != 'S') {
        fprintf(stderr, "threshold type error!\nr for correlation threshold\ns for spasity threshold\n");
        return 1;
    }
    const bool save_cormat = (save == 'y' || save == 'Y');
    std::vector<float> thr;
    for (int q = a + 4; q < argc; q++) thr.push_back((float)atof(argv[q]));
    if (rmode && !thr.empty()) {  // the smallest r threshold goes first (CorMat.cpp:176-182)
        size_t mi = 0;
        for (size_t q = 0; q < thr.size(); q++)
            if (thr[q] < thr[mi]) mi = q;
        std::swap(thr[0], thr[mi]);
    }

    std::string err;
    pgio::Nifti mask;
    if (!pgio::read_nifti(mask_path, mask, err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    const long long V = (long long)mask.dims[0] * mask.dims[1] * mask.dims[2];
    std::vector<long long> vox;
    for (long long k = 0; k < V; k++)
        if (mask.data[k] >= prob_cut) vox.push_back(k);
    const int N = (int)vox.size();
    printf("Data size: %dx%dx%d, Grey voxel count: %d.\n", mask.dims[0], mask.dims[1], mask.dims[2], N);
    std::string mask_name = mask_path.substr(mask_path.find_last_of("/\\") + 1);
    std::vector<std::string> files = pgio::list_dir(dir, ".nii", "mask.nii");
    printf("%zu file(s) to be processed.\n", files.size());
    pg_ctx* ctx = pgio::open_ctx();
    const long long M1 = (long long)N * (N - 1) / 2;
    pg_cohort* cohort = nullptr;
    if (average) pgio::check(ctx, pg_cohort_create(ctx, N, avg_kind == 'f', kWeighted, &cohort), "pg_cohort_create");
    size_t subjects = 0;
    for (const std::string& fn : files) {
        std::string path = pgio::join(dir, fn);
        if (path == mask_path) continue;
        pgio::Nifti img;
        if (!pgio::read_nifti(path, img, err)) {
            fprintf(stderr, "%s\n", err.c_str());
            if (average) return 1;   // the average would silently lose a subject
            continue;
        }
        if ((long long)img.dims[0] * img.dims[1] * img.dims[2] != V) {
            fprintf(stderr, "%s: volume size differs from the mask\n", path.c_str());
            if (average) return 1;
            continue;
        }
        const int T = img.T;
        // BOLD[l*N + i] (CorMat.cpp:208-231)
        std::vector<float> bold((size_t)T * N);
        for (int l = 0; l < T; l++)
            for (int i = 0; i < N; i++) bold[(size_t)l * N + i] = img.data[(size_t)l * V + vox[i]];
        printf("\ncalculating correlation for %s ... BOLD length: %d\n", path.c_str(), T);
        if (average) {
            pgio::check(ctx, pg_cohort_add(ctx, cohort, bold.data(), T, 0), "pg_cohort_add");
            subjects++;
        }
        if (!per_subject) continue;
        const std::string out_base = pgio::stem(path) + "_" + std::to_string(N);
        if (save_cormat) {
            std::vector<float> r((size_t)std::max(M1, 1LL));
            pgio::check(ctx, pg_correlation_packed(ctx, bold.data(), N, T, kWeighted, 0, r.data()), "correlation");
            pgio::write_cormat(out_base + ".cormat", r.data(), M1);
        }
        for (float t : thr) {
            pg_build_opts o;
            pg_build_opts_default(&o);
            o.weighted = kWeighted;
            o.precision = PG_SPLIT_BF16;
            if (const char* e = getenv("PAGANI_PRECISION")) o.precision = strcmp(e, "fp32") == 0 ? PG_FP32 : PG_SPLIT_BF16;
            float s_out, r_out;
            if (rmode) {
                o.mode = PG_THRESH_R;
                // weighted tool: r > r_thresh - 1e-6 in float (W CorMat.cpp:310)
                o.value = kWeighted ? (double)(float)((double)t - 1e-6) : (double)t;
            } else {
                o.mode = PG_THRESH_SPARSITY;
                o.value = t;
            }
            pg_graph* g = nullptr;
            pg_build_info info;
            pgio::check(ctx, pg_build_graph(ctx, bold.data(), N, T, &o, &g, &info), "pg_build_graph");
            pgio::Csr c = pgio::download(ctx, g);
            pg_graph_free(g);
            if (rmode) {
                r_out = t;
                s_out = (float)(100.0 * (double)c.C.size() / (double)M1 / 2);   // CorMat.cpp:304
            } else {
                s_out = t;
                r_out = (float)info.tau;
                printf("threshold for sparsity = %g\ncorresponding r_threshold = %g\n", (double)t, info.tau);
            }
            char suffix[64];
            snprintf(suffix, sizeof suffix, "_spa%.3f%%_cor%.3f", (double)s_out, (double)r_out);
            std::string out = out_base + suffix + (kWeighted ? "_weighted.csr" : ".csr");
            printf("generating %s...\n", out.c_str());
            if (!pgio::write_csr(out, c)) fprintf(stderr, "cannot write %s\n", out.c_str());
        }
    }
    if (average && subjects > 0) {
        const std::string out_base = cohort_base(dir, subjects, N);
        printf("\naveraging %zu subject(s) (%s)\n", subjects, avg_kind == 'f' ? "Fisher z" : "plain r");
        if (save_cormat) {
            std::vector<float> r((size_t)std::max(M1, 1LL));
            pgio::check(ctx, pg_cohort_packed(ctx, cohort, r.data()), "pg_cohort_packed");
            pgio::write_cormat(out_base + ".cormat", r.data(), M1);
        }
        for (float t : thr) {
            pg_graph* g = nullptr;
            pg_build_info info;
            pgio::check(ctx, pg_cohort_graph(ctx, cohort, rmode ? PG_THRESH_R : PG_THRESH_SPARSITY, (double)t, &g, &info),
                        "pg_cohort_graph");
            pgio::Csr c = pgio::download(ctx, g);
            pg_graph_free(g);
            const float s_out = rmode ? (float)(100.0 * (double)c.C.size() / (double)M1 / 2) : t;
            const float r_out = rmode ? t : (float)info.tau;
            char suffix[64];
            snprintf(suffix, sizeof suffix, "_spa%.3f%%_cor%.3f", (double)s_out, (double)r_out);
            std::string out = out_base + suffix + ".csr";
            printf("generating %s...\n", out.c_str());
            if (!pgio::write_csr(out, c)) fprintf(stderr, "cannot write %s\n", out.c_str());
        }
    }
    if (cohort) pg_cohort_free(cohort);
    pg_destroy(ctx);
    return 0;
}
