/*
 * ref_driver.cpp -- extern "C" entry points onto the reference's OWN CPU
 * functions, compiled unmodified from the reference tree by oracle/Makefile
 * into oracle/_ref/.  Test infrastructure only (the checker that pins the
 * oracle restatement, and the "reference" CPU baseline in bench.py).
 *
 * One shared object is built per reference translation-unit group because the
 * groups define clashing global names (FormFullGraph, CorMat_cpu, ...).  The
 * group is selected with -DREF_GROUP_<NAME>.
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#if defined(REF_GROUP_CUCORMAT)
/* U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp */
long long FormFullGraph(bool* adjacent, float* Cormat, int N, float threshold);
float FormFullGraph_s(bool* adjacent, float* Cormat, int N, long long threshold);
void FormCSRGraph(int* R, int* C, bool* adjacent, int N);
void CorMat_cpu(float* Cormat, float* BOLD, int N, int L);
void post_block(float* Cormat, float* Cormat_blocked, int N, int block_size, bool fishtran_flag);
float inv_fisher_trans(float z);
/* main() of CorMat.cpp references the GPU routines; they are never reached
 * through this driver. */
int CorMat_gpu(float*, float*, int, int, int) { return -1; }
long long find_max(float*, long long) { return 0; }
float select_GPU(float*, long long, long long) { return 0.0f; }

extern "C" {
void ref_cormat_cpu(float* cormat, float* bold, int N, int L) { CorMat_cpu(cormat, bold, N, L); }
long long ref_form_graph_r(float* cormat, int N, float thr, int* R, int* C, long long cap)
{
    std::vector<char> adj((size_t)N * N);
    long long nnz = FormFullGraph((bool*)adj.data(), cormat, N, thr);
    if (nnz > cap) return -1;
    FormCSRGraph(R, C, (bool*)adj.data(), N);
    return nnz;
}
long long ref_form_graph_s(float* cormat, int N, long long k, int* R, int* C, float* tau, long long cap)
{
    if (2 * k > cap) return -1;
    std::vector<char> adj((size_t)N * N);
    *tau = FormFullGraph_s((bool*)adj.data(), cormat, N, k);
    FormCSRGraph(R, C, (bool*)adj.data(), N);
    return (long long)R[N];
}
/* One subject of the averaging branch (CorMat.cpp:466-469): post_block adds
 * r or fisher_trans(r).  The packed r are laid out as a single N x N block
 * (block_size = N), so post_block's block arithmetic maps (i, j) to i*N + j. */
void ref_cohort_add(float* cormat, const float* r_packed, int N, int fisher)
{
    std::vector<float> blocked((size_t)N * N, 0.0f);
    long long k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) blocked[(size_t)i * N + j] = r_packed[k++];
    post_block(cormat, blocked.data(), N, N, fisher != 0);
}
/* The end of the branch, restated from main() (CorMat.cpp:514-524), with the
 * reference's own inv_fisher_trans. */
void ref_cohort_finish(float* cormat, long long M1, int files, int fisher)
{
    for (long long i = 0; i < M1; i++) {
        cormat[i] /= files;
        if (fisher) cormat[i] = inv_fisher_trans(cormat[i]);
    }
}
}
#elif defined(REF_GROUP_CORMAT_CPU)
/* U/CorMat/CorMat_CPU/CorMat/CorMat_CPU.cpp */
extern int numThread;
void CorMat_cpu_MT(float* Cormat, float* BOLD, int N, int L);
int FormFullGraph(bool* adjacent, float* Cormat, int N, float threshold);
void FormCSRGraph(int* R, int* C, bool* adjacent, int N);
extern "C" {
void ref_cormat_cpu_mt(float* cormat, float* bold, int N, int L, int threads)
{
    numThread = threads;
    CorMat_cpu_MT(cormat, bold, N, L);
}
long long ref_form_graph_abs(float* cormat, int N, float thr, int* R, int* C, long long cap)
{
    std::vector<char> adj((size_t)N * N);
    long long nnz = FormFullGraph((bool*)adj.data(), cormat, N, thr);
    if (nnz > cap) return -1;
    FormCSRGraph(R, C, (bool*)adj.data(), N);
    return nnz;
}
}
#elif defined(REF_GROUP_METRICS)
/* U/BC/BC_CPU/BC_CPU/BC_CPU.cpp, U/Cp/Cp/Cp.cpp, U/BFS_MulCPU/BFS_MulCPU/APSP_BFS.cpp,
 * U/cuda_EC/cuda_EC/Modularity_CPU.cpp */
void Betweenness_CPU(int* row, int* col, int numVertices, int numEdges, float* BC);
double Cp(int* C, int* R, float* Cp, int N);
double APSP_BFS(float* APSP_output, int* row, int* col, const int numVertices);
void Partition(int* R, int* C, int* Result);
extern long long N, Ntemp, seed;
extern double *v, *v0, *verr, *vv, *sumBG;
float* Li_result;  /* defined by MUBFS_LP_main.cpp in the tool */
/* Partition() allocates NewRow with N ints and writes N+1 of them
 * (Modularity_CPU.cpp:64,90-107; the GPU twin allocates N+1,
 * modularity_GPU.cu:432).  MSVC's heap tolerated the one-int overrun; here
 * every array allocation of this group gets a little slack instead. */
#include <new>
void* operator new[](size_t sz) { void* p = std::malloc(sz + 64); if (!p) throw std::bad_alloc(); return p; }
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, size_t) noexcept { std::free(p); }
/* Timer.h functions used by Modularity_CPU.cpp (timing only). */
void Setup(int) {}
void Start(int) {}
void Stop(int) {}
void Reset(int) {}
double GetElapsedTime(int) { return 0.0; }
void PrintTime(int) {}
/* Maslov() is declared by Modularity_CPU.cpp but only main() of the GPU
 * tool calls it. */
void Maslov(int*, int*, int*, int*, int, int) {}

extern "C" {
void ref_betweenness(int* R, int* C, int n, int nnz, float* bc) { Betweenness_CPU(R, C, n, nnz, bc); }
double ref_cp(int* R, int* C, int n, float* cp) { return Cp(C, R, cp, n); }
double ref_apsp_bfs(int* R, int* C, int n, float* li)
{
    std::vector<float> apsp((size_t)n * n);
    Li_result = li;
    return APSP_BFS(apsp.data(), R, C, n);
}
void ref_partition(int* R, int* C, int n, int* result)
{
    N = n;
    std::vector<double> a(n), b(n), c(n), d(n), e(n);
    v = a.data(); v0 = b.data(); vv = c.data(); verr = d.data(); sumBG = e.data();
    seed = 0;
    Partition(R, C, result);
}
}
#elif defined(REF_GROUP_WEIGHTED)
/* W/Cp/Cp/Cp_2.cpp, W/Lp/CUBFW_Lp/CUBFW_Lp/BFW.cpp, W/Lp/CUBFW_Lp/CUBFW_Lp/FormBlock.cpp */
double Cp_2(int* C, int* R, float* V, float* Cp, int N);
void BFW_C(float* costmat, long long numVertices, long long block_size);
void init_block(float* costmat, const int* row, const int* col, const float* power,
                const int numVertices, const int block_size);
extern "C" {
double ref_cp2(int* R, int* C, float* V, int n, float* cp) { return Cp_2(C, R, V, cp, n); }
/* Dense blocked FW of the reference on a graph padded to a multiple of
 * block; returns the n x n row-major distance matrix. */
void ref_bfw(int* R, int* C, float* V, int n, int block, float* dist_out)
{
    int np = (n + block - 1) / block * block;
    std::vector<int> rp(np + 1);
    for (int i = 0; i <= n; i++) rp[i] = R[i];
    for (int i = n + 1; i <= np; i++) rp[i] = R[n];
    std::vector<float> cm((size_t)np * np);
    init_block(cm.data(), rp.data(), C, V, np, block);
    BFW_C(cm.data(), np, block);
    int cnt = np / block;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            long long off = ((long long)(i / block) * cnt + j / block) * block * block;
            dist_out[(long long)i * n + j] = cm[off + (i % block) * block + (j % block)];
        }
}
}
#elif defined(REF_GROUP_WCORMAT)
/* W/CorMat/CUCorMat/CUCorMat/CorMat.cpp */
long long FormFullGraph(bool* adjacent, float* Cormat, int N, float threshold);
float FormFullGraph_s(bool* adjacent, float* Cormat, int N, long long threshold);
void FormCSRGraph(int* R, int* C, float* V, bool* adjacent, int N, float* Cormat);
void post_block(float* Cormat, float* Cormat_blocked, int N, int block_size, bool fishtran_flag);
float inv_fishertrans(float z);
int CorMat_gpu(float*, float*, int, int, int) { return -1; }
long long find_max(float*, long long) { return 0; }
float select_GPU(float*, long long, long long) { return 0.0f; }
extern "C" {
/* main() passes r_thresh[k] - ep to the float parameter (CorMat.cpp:310). */
long long ref_wform_graph_r(float* cormat, int N, float thr, int* R, int* C, float* V, long long cap)
{
    std::vector<char> adj((size_t)N * N);
    long long nnz = FormFullGraph((bool*)adj.data(), cormat, N, (float)(thr - 1e-6));
    if (nnz > cap) return -1;
    FormCSRGraph(R, C, V, (bool*)adj.data(), N, cormat);
    return nnz;
}
/* The weighted tool's averaging branch: post_block with its range rule
 * (-1-ep, 1+ep) and fishertrans (W CorMat.cpp:466-469, :826-852), then the
 * division and inv_fishertrans of main() (:514-524). */
void ref_wcohort_add(float* cormat, const float* r_packed, int N, int fisher)
{
    std::vector<float> blocked((size_t)N * N, 0.0f);
    long long k = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) blocked[(size_t)i * N + j] = r_packed[k++];
    post_block(cormat, blocked.data(), N, N, fisher != 0);
}
void ref_wcohort_finish(float* cormat, long long M1, int files, int fisher)
{
    for (long long i = 0; i < M1; i++) {
        cormat[i] /= files;
        if (fisher) cormat[i] = inv_fishertrans(cormat[i]);
    }
}
}
#elif defined(REF_GROUP_WNEWMAN)
/* W/Newman_Modularity_GPU/CUmodularity/Modularity_CPU.cpp: the weighted
 * tool's CPU Partition, which reads the edge values through the global Vf
 * (defined by modularity_GPU.cu in the tool, here by the caller). */
void Partition(int* R, int* C, int* Result);
extern long long N, Ntemp, seed;
extern double *v, *v0, *verr, *vv, *sumBG;
float* Vf;
#include <new>
void* operator new[](size_t sz) { void* p = std::malloc(sz + 64); if (!p) throw std::bad_alloc(); return p; }
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, size_t) noexcept { std::free(p); }
void Setup(int) {}
void Start(int) {}
void Stop(int) {}
void Reset(int) {}
double GetElapsedTime(int) { return 0.0; }
void PrintTime(int) {}
void Maslov(int*, int*, int*, int*, int, int) {}
extern "C" {
void ref_wpartition(int* R, int* C, float* V, int n, int* result)
{
    N = n;
    std::vector<double> a(n), b(n), c(n), d(n), e(n);
    v = a.data(); v0 = b.data(); vv = c.data(); verr = d.data(); sumBG = e.data();
    seed = 0;
    Vf = V;
    Partition(R, C, result);
}
}
#elif defined(REF_GROUP_MASLOV) || defined(REF_GROUP_WMASLOV)
/* U/cuda_EC/cuda_EC/Maslov.cpp (Maslov, Rewire) or W/Maslov/Maslov/Maslov.cpp
 * (Maslov_weighted_1), compiled with ref_shim/seeded_rand.h forced in. */
extern "C" {
unsigned int ref_rand_seed = 1;
static unsigned int ref_lcg_state = 1;
int ref_rand15(void)
{
    ref_lcg_state = ref_lcg_state * 214013u + 2531011u;
    return (int)((ref_lcg_state >> 16) & 0x7fff);
}
void ref_srand15(unsigned int seed) { ref_lcg_state = seed; }
}
#if defined(REF_GROUP_MASLOV)
void Maslov(int* R_dst, int* C_dst, int* R_src, int* C_src, int Rlength, int Clength);
extern "C" void ref_maslov(int* R_src, int* C_src, int N, int nnz, unsigned int seed, int* R_dst, int* C_dst)
{
    ref_rand_seed = seed;
    Maslov(R_dst, C_dst, R_src, C_src, N + 1, nnz);
}
#else
void Maslov_weighted_1(int* R_dst, int* C_dst, float* V_dst, int* R_src, int* C_src, float* V_src, int Rlength,
                       int Clength);
extern "C" void ref_wmaslov(int* R_src, int* C_src, float* V_src, int N, int nnz, unsigned int seed, int* R_dst,
                            int* C_dst, float* V_dst)
{
    ref_rand_seed = seed;
    Maslov_weighted_1(R_dst, C_dst, V_dst, R_src, C_src, V_src, N + 1, nnz);
}
#endif

#else
#error "select a reference group with -DREF_GROUP_<NAME>"
#endif
