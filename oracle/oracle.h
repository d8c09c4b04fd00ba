/*
 * oracle.h -- CPU restatement of the PAGANI hot path, used ONLY as test
 * infrastructure (the checker): tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py.  Nothing in the product library
 * (libpagani) links or calls this code.
 *
 * Arithmetic conventions (shared with the CUDA kernels so that results can be
 * compared bit for bit where the text says "exact"):
 *   - z-score in FP64: mean = (sum_t x_t) / T with sequential adds, then
 *     s = sqrt(sum_t (x_t - mean)^2) with each square rounded before the add,
 *     z_t = (x_t - mean) / s.  A zero-variance row becomes the zero vector.
 *   - r(i,j) = sum_t z_i[t] * z_j[t], t ascending, each term added with one
 *     fused multiply-add (r = fma(z_i[t], z_j[t], r), a single rounding, as
 *     the reference's SGEMM accumulates).  Everything else is compiled with
 *     -ffp-contract=off, so no other multiply-add is fused.
 *   - the reference's range rule (post_block): an r outside [-1, 1]
 *     (unweighted) or outside (-1-1e-6, 1+1e-6) (weighted) is stored as 0.
 */
#ifndef PAGANI_ORACLE_H
#define PAGANI_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

int     or_zscore(const float* bold_TxN, int N, int T, double* z_NxT);
double  or_pair_r(const double* z, int T, int i, int j, int weighted);
void    or_corr_packed(const double* z, int N, int T, int weighted, double* r_packed);
int64_t or_sparsity_k(int N, float s_percent);
float   or_weighted_r_threshold(float thr);
int64_t or_graph_r(const double* r_packed, int N, double thr, int abs_mode,
                   int32_t* R, int32_t* C, float* V, int64_t cap);
int64_t or_graph_k(const double* r_packed, int N, int64_t k, int abs_mode, double* tau,
                   int32_t* R, int32_t* C, float* V, int64_t cap);
void    or_degree(const int32_t* R, const float* V, int N, float* deg, int32_t* isolated);
void    or_cp_binary(const int32_t* R, const int32_t* C, int N, int64_t* tri, float* cp, double* mean);
void    or_onnela(const int32_t* R, const int32_t* C, const float* V, int N, int vmax_first_n,
                  float* cp, double* mean);
int     or_bfs_paths(const int32_t* R, const int32_t* C, int N, double* inv_sum,
                     int64_t* hop_hist, int max_hop, double* lp);
int     or_bfs_source(const int32_t* R, const int32_t* C, int N, int s, int32_t* dist, int64_t* sigma);
void    or_brandes(const int32_t* R, const int32_t* C, int N, double* bc);
void    or_fw_dense(float* d, int n);
int     or_weighted_paths(const int32_t* R, const int32_t* C, const float* V, int N,
                          float* eff, double* lp);
int     or_newman(const int32_t* R, const int32_t* C, int N, int gpu_rule_above,
                  int32_t* labels, double* Q, int* n_modules, int* n_rounds);
int     or_newman_weighted(const int32_t* R, const int32_t* C, const float* Vw, int64_t wn, int N,
                           int gpu_rule_above, int32_t* labels, double* Q, int* n_modules, int* n_rounds);
int64_t or_maslov(const int32_t* R, const int32_t* C, const float* V, int N, uint64_t seed,
                  int64_t attempts, int32_t* R_out, int32_t* C_out, float* V_out);
int64_t or_rewire_seq(const int32_t* R, const int32_t* C, const float* V, int N, uint32_t seed, int64_t attempts,
                      int32_t* R_out, int32_t* C_out, float* V_out);
int     or_eigen_centrality(const int32_t* R, const int32_t* C, const float* V, int N, int raw,
                            double* ec, double* eigenvalue, double* residual);
double  or_ln(double x);
double  or_exp(double x);
double  or_fisher(double r);
double  or_inv_fisher(double z);
void    or_cohort_add(const double* z, int N, int T, int weighted, int fisher, double* acc);
void    or_cohort_finish(const double* acc, int64_t M1, int subjects, int fisher, double* key);
int     or_participation(const int32_t* R, const int32_t* C, const float* V, int N, const float* module,
                         float* pc, float* pc_norm);

#ifdef __cplusplus
}
#endif
#endif
