/*
 * pagani.h -- C ABI of the B200-native PAGANI hot path (libpagani.so).
 *
 * The reference has no library API: its boundary is a set of console tools
 * that exchange .nii/.csr/.nm files, and inside each tool a C function with
 * host pointers does the work.  Every entry point below names the reference
 * function it replaces (paths relative to the reference project root,
 *   U/ = src/BNAPlatform-win64-cuda7.0-20151118/src/,
 *   W/ = src/BNAPlatform-weighted-network-win64-cuda7.0-20151118/src/).
 *
 * Conventions
 *   - every call returns pg_status and never exits, blocks on stdin or
 *     prints; pg_last_error() holds the message of the last failure;
 *   - plain pointers and sizes only; host pointers unless a flag says the
 *     pointer is device memory of the context's GPU;
 *   - one pg_ctx per host thread; a context owns one CUDA stream and a
 *     device workspace that is reused across calls;
 *   - graphs (pg_graph) are device-resident CSR: row offsets R[n+1],
 *     ascending column indices C[nnz], optional float weights V[nnz];
 *     undirected graphs store both directions and no self loops, exactly
 *     as the reference .csr format (manual p10).
 */
#ifndef PAGANI_H
#define PAGANI_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PG_OK = 0,
    PG_ERR_INVALID = 1,       /* bad argument */
    PG_ERR_CUDA = 2,          /* CUDA runtime error (message in pg_last_error) */
    PG_ERR_NOMEM = 3,         /* device allocation failed */
    PG_ERR_TOO_LARGE = 4,     /* result does not fit the 32-bit CSR format */
    PG_ERR_INTERNAL = 5,      /* an internal consistency check failed */
    PG_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up */
    PG_ERR_NO_DEVICE = 7      /* no usable sm_100 device */
} pg_status;

typedef struct pg_ctx pg_ctx;
typedef struct pg_graph pg_graph;

typedef enum { PG_THRESH_R = 0, PG_THRESH_SPARSITY = 1 } pg_thresh_mode;
typedef enum { PG_SIGNED = 0, PG_ABS = 1 } pg_sign;
typedef enum { PG_FP32 = 0, PG_SPLIT_BF16 = 1 } pg_precision;

/* ------------------------------------------------------------- context */
pg_status   pg_create(pg_ctx** ctx, int device);
pg_status   pg_destroy(pg_ctx* ctx);
const char* pg_last_error(const pg_ctx* ctx);
const char* pg_status_string(pg_status s);
pg_status   pg_synchronize(pg_ctx* ctx);
/* The cudaStream_t the context issues its work on. */
void*       pg_stream(pg_ctx* ctx);
/* Number of kernel launches issued by this context so far. */
int64_t     pg_launch_count(const pg_ctx* ctx);
/* Per-kernel device time, for measurement harnesses (no counterpart in the
 * reference).  With profiling on, the library records CUDA events on the
 * context stream around every launch of its dominant kernels ("k_brandes",
 * "k_bc_dense"); pg_profile_get returns the launches and summed milliseconds
 * of one kernel since the last reset (it synchronises the stream).  Off by
 * default; the events cost a few microseconds per launch. */
pg_status   pg_profile_enable(pg_ctx* ctx, int32_t on);
pg_status   pg_profile_reset(pg_ctx* ctx);
pg_status   pg_profile_get(pg_ctx* ctx, const char* kernel, int64_t* launches, double* ms);
/* Failure-path test hook (no counterpart in the reference): the next
 * split-BF16 tensor-core Gram launch of this context makes its TMA producer
 * wait wait_ns on a barrier that nothing arrives on, before it issues any
 * copy; the wait runs out, every warp of the kernel gives up, TMEM is freed
 * and the call (pg_build_graph) returns PG_ERR_TIMEOUT.  The context stays
 * usable.  Applies to one launch; 0 clears it. */
pg_status   pg_debug_stall_next_gram(pg_ctx* ctx, uint64_t wait_ns);

/* ------------------------------------------------------------- graphs */
/* Replaces the .csr reads of every metric tool (e.g. U/Cp/Cp/Cp_main.cpp:107-116,
 * W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp_main.cpp:100-118).  V may be NULL
 * (binary graph).  on_device != 0: R/C/V are device pointers. */
pg_status pg_graph_from_csr(pg_ctx* ctx, const int32_t* R, const int32_t* C, const float* V,
                            int32_t n, int64_t nnz, int32_t on_device, pg_graph** out);
pg_status pg_graph_info(const pg_graph* g, int32_t* n, int64_t* nnz, int32_t* weighted);
/* Copy the CSR out (host or device buffers sized n+1 / nnz / nnz). */
pg_status pg_graph_to_csr(pg_ctx* ctx, const pg_graph* g, int32_t* R, int32_t* C, float* V,
                          int32_t on_device);
pg_status pg_graph_free(pg_graph* g);

/* ------------------------------------------------- network construction */
typedef struct {
    int32_t mode;            /* pg_thresh_mode */
    double  value;           /* r threshold (edge iff key > value) or sparsity in percent */
    int32_t sign;            /* pg_sign: key = r (GPU tool) or |r| (CorMat_CPU) */
    int32_t precision;       /* pg_precision of the Gram tiles */
    int32_t weighted;        /* store V = key, weighted range rule (-1-1e-6, 1+1e-6) */
    double  guard;           /* half-width of the FP64 recheck band around the threshold */
    int32_t input_on_device; /* bold is a device pointer */
    int32_t exact_weights;   /* weighted: V recomputed in FP64 for every edge */
} pg_build_opts;

typedef struct {
    double  tau;             /* threshold actually applied (k-th key in sparsity mode) */
    int64_t edges;           /* undirected edges kept */
    int64_t band_pairs;      /* pairs decided by the FP64 recheck */
    int64_t above_pairs;     /* pairs decided by the Gram tile alone */
    int32_t zero_variance;   /* voxels with zero variance (their r is 0) */
    double  sparsity_percent;/* 100 * edges / M1 */
    double  ms_zscore, ms_hist, ms_emit, ms_select, ms_csr; /* device time per stage */
    double  band_err_max;    /* max |r_tile - r| over the band pairs (r: FP64 recheck) */
    double  band_err_mean;   /* mean of the same */
} pg_build_info;

/* Defaults: r mode 0.3, signed, split-BF16, binary, guard 2e-3, host input. */
void pg_build_opts_default(pg_build_opts* o);

/* Network construction of CUCorMat: replaces CorMat_gpu (U/CorMat/CUCorMat/
 * CUCORMAT/CorMat.cu:18) + post_block (CorMat.cpp:775) + FormFullGraph (:633)
 * / select + FormFullGraph_s (:655-773) + FormCSRGraph (:839); weighted
 * variant W/CorMat/CUCorMat/CUCorMat/CorMat.cpp:647-882.  bold is time-major
 * T x N float32 (BOLD[t*N + i], CorMat.cpp:208-231).  The correlation matrix
 * is never materialised.  The edge set equals the FP64 oracle's: r is
 * decided from the tensor/FP32 tile unless it lies within `guard` of the
 * threshold (or of +-1), in which case it is recomputed in FP64. */
pg_status pg_build_graph(pg_ctx* ctx, const float* bold, int32_t N, int32_t T,
                         const pg_build_opts* opts, pg_graph** out, pg_build_info* info);

/* Number of undirected edges for a sparsity of s percent, as CUCorMat's
 * main() computes it (CorMat.cpp:310-312). */
int64_t pg_sparsity_edges(int32_t N, float s_percent);

/* Packed upper-triangle r (M1 = N(N-1)/2 floats, row-major i<j): the
 * .cormat payload written when save_cormat = y (CorMat.cpp:285-294).
 * r is rounded from the FP64 value. Output is a host buffer. */
pg_status pg_correlation_packed(pg_ctx* ctx, const float* bold, int32_t N, int32_t T,
                                int32_t weighted, int32_t input_on_device, float* r_packed);

/* ------------------------------------------------------ cohort averaging */
/* Subject-averaged graphs: the to_average modes of CUCorMat (argv[3] = yn,
 * yf, bn, bf), U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:380-620 and
 * W/CorMat/CUCorMat/CUCorMat/CorMat.cpp:386-620.  The reference adds each
 * subject's r (n) or fisher_trans(r) (f, :35-41) into a float matrix in
 * post_block (:775-838), divides by the subject count and applies
 * inv_fisher_trans (:514-524).  Here the sum is FP64 and device-resident
 * (N(N-1)/2 doubles), r is the exact FP64 r of pg_build_graph's recheck,
 * and ln/exp are evaluated so that the averaged keys are bit-identical to
 * the FP64 oracle's.  weighted != 0 selects the weighted tool: its range
 * rule (-1-1e-6, 1+1e-6) and edge values V = float(average). */
typedef struct pg_cohort pg_cohort;
pg_status pg_cohort_create(pg_ctx* ctx, int32_t N, int32_t fisher, int32_t weighted, pg_cohort** out);
/* Adds one subject: bold is time-major T x N float32 (host, or device when
 * input_on_device != 0); subjects may differ in T. */
pg_status pg_cohort_add(pg_ctx* ctx, pg_cohort* c, const float* bold, int32_t T, int32_t input_on_device);
/* Thresholds the current average once: mode PG_THRESH_R keeps key > value
 * (FormFullGraph, CorMat.cpp:633, signed, no 1e-6 shift in either tool's
 * averaged branch), PG_THRESH_SPARSITY keeps the top pg_sparsity_edges(N, value)
 * keys with the reference's tie rule (FormFullGraph_s, :693-773).  info: tau,
 * edges, sparsity_percent and stage times. */
pg_status pg_cohort_graph(pg_ctx* ctx, pg_cohort* c, int32_t mode, double value, pg_graph** out,
                          pg_build_info* info);
/* The averaged matrix as the .cormat payload (CorMat.cpp:534-543): M1 floats,
 * packed upper triangle, row-major i < j; host buffer. */
pg_status pg_cohort_packed(pg_ctx* ctx, pg_cohort* c, float* r_packed);
pg_status pg_cohort_info(const pg_cohort* c, int32_t* N, int32_t* subjects);
pg_status pg_cohort_free(pg_cohort* c);

/* -------------------------------------------------------------- metrics */
/* Degree (U/Degree/Degree/Degree.cpp:85-91) or strength for weighted graphs
 * (W/Degree/Degree/Degree.cpp:82-88).  deg: host float[n]. */
pg_status pg_degree(pg_ctx* ctx, const pg_graph* g, float* deg, int32_t* isolated);

/* Clustering coefficient.  kind 0: binary, Cp (U/Cp/Cp/Cp.cpp:21-116);
 * triangles (int64[n], optional) are exact.  kind 1: Onnela weighted,
 * Cp_2 (W/Cp/Cp/Cp_2.cpp:23-130); flags bit 0 = take the weight maximum over
 * V[0..n) only, as the reference CPU does.  cp: host float[n]; mean over all
 * n nodes. */
pg_status pg_clustering(pg_ctx* ctx, const pg_graph* g, int32_t kind, int32_t flags,
                        float* cp, int64_t* triangles, double* mean);

/* Allocation-free binary clustering (no counterpart in the reference).  For
 * callers that cannot allocate device memory -- a host whose GPU memory is
 * owned by another component (a framework's caching allocator, a plugin host
 * that reserves the device at start-up) or a latency-critical pipeline that
 * forbids cudaMalloc after initialisation because it can synchronise the
 * device.  R/C (the CSR, n+1 and R[n] entries), cp (float[n]) and
 * triangles (int64[n], may be NULL) are DEVICE pointers owned by the caller;
 * work is issued on `stream` (a cudaStream_t, NULL = legacy default stream)
 * and is not waited for.  Scratch is a 16 MiB static device array inside the
 * library, and the neighbour bitmap of a node (n bits) lives in shared memory:
 * n is limited to pg_clustering_noalloc_max_nodes(), the smaller of the
 * array's 2,097,150 nodes and the bitmap's limit on the current device
 * (1,826,816 nodes on a B200); larger n returns PG_ERR_TOO_LARGE.  Every GPU
 * that loads the library holds the array until exit, and calls that overlap
 * on the GPU race on it.  The first call on a device (and the first call after
 * cudaDeviceReset gives the device a new context) resolves the array's device
 * address and caches the SM count and shared-memory limit, with that device
 * current; make that first call before any stream capture.  No
 * cudaMalloc/cudaFree. */
pg_status pg_clustering_noalloc(const int32_t* R, const int32_t* C, int32_t n, float* cp, int64_t* triangles,
                                void* stream);
int64_t   pg_clustering_noalloc_max_nodes(void);

/* Hop path length and nodal efficiency: APSP_BFS (U/BFS_MulCPU/BFS_MulCPU/
 * APSP_BFS.cpp:27-147).  eff[i] = sum_j 1/d_ij / (n-1) (float, optional),
 * inv_sum[i] = sum_j 1/d_ij (double, optional), lp = n(n-1)/sum_ij 1/d_ij,
 * hop_hist[d] = ordered pairs at distance d for d <= max_hop (optional),
 * diameter = largest finite distance. */
pg_status pg_paths(pg_ctx* ctx, const pg_graph* g, float* eff, double* inv_sum, double* lp,
                   int64_t* hop_hist, int32_t max_hop, int32_t* diameter);

/* Brandes betweenness from all sources: replaces CUBC (U/BC/CUBC/CUBC.cpp:13)
 * and Betweenness_CPU (U/BC/BC_CPU/BC_CPU/BC_CPU.cpp:6).  Sum over ordered
 * source/target pairs, as the reference.  Path counts are exact int64,
 * dependencies FP64.  bc: host float[n] (optional), bc64: host double[n]
 * (optional).  When eff/lp are given, the hop path length of pg_paths is
 * produced from the same BFS sweep. */
pg_status pg_betweenness(pg_ctx* ctx, const pg_graph* g, float* bc, double* bc64,
                         float* eff, double* lp);

/* Exact single-source hop distances (-1 = unreachable) and shortest-path
 * counts for ns sources: dist int32[ns*n], sigma int64[ns*n] (host). */
pg_status pg_bfs_sigma(pg_ctx* ctx, const pg_graph* g, const int32_t* sources, int32_t ns,
                       int32_t* dist, int64_t* sigma);

/* Weighted path length by blocked Floyd-Warshall on d = 1/w: CUBFW_Lp
 * (W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp.cpp:13-162, cuAPSP CUBFW.cpp:19).
 * dist: host float[n*n] (optional, row-major), eff: host float[n], lp. */
pg_status pg_fw_paths(pg_ctx* ctx, const pg_graph* g, float* dist, float* eff, double* lp);

/* Batched weighted path length + Onnela clustering for many small graphs in
 * grouped launches (one FW sweep over all graphs).  eff and cp are
 * concatenated per graph (sum of n floats each); lp and cp_mean per graph. */
pg_status pg_fw_batched(pg_ctx* ctx, const pg_graph* const* graphs, int32_t count,
                        float* eff, double* lp, float* cp, double* cp_mean);

/* Newman leading-eigenvector modularity: Partition_GPU / Sub_Partition_GPU /
 * Lead_Vector_GPU (U/cuda_EC/cuda_EC/modularity_GPU.cu:230-530) with the CPU
 * variant's rules for sub-graphs of at most gpu_rule_above nodes
 * (Modularity_CPU.cpp:48-298).  labels: host int32[n] numbered from 1 in
 * division order; Q in FP64.  log (optional) receives one line per round. */
typedef void (*pg_log_fn)(const char* line, void* user);
pg_status pg_newman(pg_ctx* ctx, const pg_graph* g, int32_t gpu_rule_above, int32_t* labels,
                    double* Q, int32_t* n_modules, pg_log_fn log, void* user);

/* The weighted Newman tool (W/Newman_Modularity_GPU/CUmodularity): the same
 * partition with edge values in the power iteration's products only; the
 * degrees, M and Q stay binary as in the reference.  The tool reads the values
 * by position in the value array of the file's graph: a sub-graph above
 * gpu_rule_above nodes multiplies its q-th edge by value q
 * (modularity_GPU.cu:135), a smaller one every term of its i-th row by value
 * i (Modularity_CPU.cpp:261); positions past the array count 0.  weights_of
 * holds that array (null: g itself; the tool passes the original graph when
 * it partitions a random surrogate).  Labels and Q as pg_newman. */
pg_status pg_newman_weighted(pg_ctx* ctx, const pg_graph* g, const pg_graph* weights_of, int32_t gpu_rule_above,
                             int32_t* labels, double* Q, int32_t* n_modules, pg_log_fn log, void* user);

/* Eigenvector centrality by the power method of the CUEC tools:
 * Lead_Vector_GPU in U/CUEC/CUEC/CUEC_unweighted.cu:61-214 (edges count 1)
 * and W/CUEC/weighted-net.cu:55-218 (a graph with weights uses them).  The
 * iteration starts from the node ids, normalises by the 2-norm each step and
 * stops when |y - u0| or |y + u0| is at most 1e-6 or after 10,000 steps.
 * raw = 0 returns the normalised vector of the last step, as the unweighted
 * tool writes it (CUEC_unweighted.cu:161); raw = 1 returns y = A x of the
 * last step, as the weighted tool writes it (weighted-net.cu:190).
 * ec: host double[n]; eigenvalue = the 2-norm of the last step's vector
 * before normalisation (the tools' _evalue.txt); iterations and residual
 * (min of the two errors) are optional. */
pg_status pg_eigen_centrality(pg_ctx* ctx, const pg_graph* g, int32_t raw, double* ec, double* eigenvalue,
                              int32_t* iterations, double* residual);

/* Participation coefficient from module labels: PC_CPU
 * (W/PC_CPU/PC_CPU/main.cpp:100-174), float arithmetic in the reference's
 * order (bit-identical).  module: host float[n] labels 1..K (the _modu.nm
 * file); edges count their weight (1 in a graph without weights).
 * pc, pc_norm: host float[n] (PC, and PC / ((K-1)/K) unless K = 1);
 * n_modules = K (optional). */
pg_status pg_participation(pg_ctx* ctx, const pg_graph* g, const float* module, float* pc, float* pc_norm,
                           int32_t* n_modules);

/* Maslov-Sneppen degree-preserving rewiring: Maslov/Rewire (U/cuda_EC/cuda_EC/
 * Maslov.cpp:8-109) and Maslov_weighted_1 (W/Maslov/Maslov/Maslov.cpp:106-196).
 * `attempts` swap attempts from a seeded counter-based generator, in rounds
 * of pg_maslov_round_size(M) attempts.  Weights stay with their edge slot. */
pg_status pg_maslov(pg_ctx* ctx, const pg_graph* g, uint64_t seed, int64_t attempts,
                    pg_graph** out, int64_t* committed);
int64_t   pg_maslov_round_size(int64_t undirected_edges);

/* Small-world ratios: gamma = Cp/<Cp_rand> (U/Cp/Cp/Cp_main.cpp:173-174),
 * lambda = Lp/<Lp_rand> (W/Lp/CUBFW_Lp/CUBFW_Lp/CUBFW_Lp_main.cpp:213-227),
 * sigma = gamma/lambda (W/SmallWorldProperty/SmallWorldProperty.cpp:188). */
pg_status pg_smallworld(double cp, const double* cp_rand, int32_t n_cp, double lp,
                        const double* lp_rand, int32_t n_lp, double* gamma, double* lambda,
                        double* sigma);

/* ------------------------------------------------------ batched subjects */
/* A cohort through the whole path in one call: the reference runs CUCorMat,
 * Degree, Cp, BFS_MulCPU / CUBC, Newman_Modularity, Maslov and
 * SmallWorldProperty as separate programs over a directory
 * (main() of U/CorMat/CUCorMat/CUCORMAT/CorMat.cpp:51,
 * U/Degree/Degree/Degree.cpp:12, U/Cp/Cp/Cp_main.cpp:28,
 * U/BC/CUBC/CUBC_main.cpp:15, U/cuda_EC/cuda_EC/modularity_GPU.cu:532 and
 * W/SmallWorldProperty/SmallWorldProperty.cpp:14); here each subject's graph stays on the device
 * while every requested metric runs.  Subjects may differ in N and T.
 * Output arrays are host buffers of N entries; NULL skips the metric.  With
 * bc set, eff and lp come from the Brandes sweep, else from pg_paths.
 * n_random > 0 adds that many Maslov surrogates per subject (swaps_per_edge x
 * edges attempts, seed pg_surrogate_seed(seed, subject, r)) and their
 * clustering and hop path length for gamma, lambda and sigma; the surrogate
 * chain is captured into a CUDA graph once per subject and replayed
 * (cuda_graphs = 0 enqueues it directly; the results are the same).
 * With build.weighted set the weighted tools' rules apply where the
 * reference has them: degree is strength (W Degree.cpp), clustering is
 * Onnela's (real graph and surrogates, W Cp_2.cpp) and modules come from
 * pg_newman_weighted (W Newman_Modularity_GPU); path length, efficiency and
 * betweenness stay hop-based (BFS_MulCPU / CUBC semantics: the weighted
 * tree's path-length tool, CUBFW_Lp, is pg_fw_paths, an N^3 computation
 * called separately). */
typedef struct {
    const float* bold;       /* T x N float32 (device pointer with build.input_on_device) */
    int32_t N, T;
    float* degree;           /* pg_degree */
    float* cp;               /* pg_clustering */
    float* eff;              /* nodal efficiency */
    float* bc;               /* pg_betweenness */
    int32_t* modules;        /* pg_newman labels */
    int64_t edges;           /* results */
    double tau, cp_mean, lp, Q;
    int32_t n_modules;
    double gamma, lambda, sigma;
    int32_t surrogate_graph_replays;   /* surrogates run as CUDA graph replays */
} pg_subject;

typedef struct {
    pg_build_opts build;
    int32_t n_random;
    int64_t swaps_per_edge;
    uint64_t seed;
    int32_t cuda_graphs;     /* replay the surrogate chain from a CUDA graph (default 1) */
} pg_run_opts;

/* Defaults: pg_build_opts_default, no surrogates, 2 swap attempts per edge
 * (U/cuda_EC/cuda_EC/Maslov.cpp:19 tries 2M), seed 1, CUDA graphs on. */
void      pg_run_opts_default(pg_run_opts* o);
uint64_t  pg_surrogate_seed(uint64_t base, int32_t subject, int32_t r);
pg_status pg_run_subjects(pg_ctx* ctx, pg_subject* subjects, int32_t n, const pg_run_opts* opts);

#ifdef __cplusplus
}
#endif
#endif
