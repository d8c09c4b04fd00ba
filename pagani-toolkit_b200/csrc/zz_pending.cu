// zz_pending.cu -- entry points whose kernels are not written yet.
#include "pg_internal.cuh"
#define PENDING(name) return pg_fail(ctx, PG_ERR_INVALID, name " is not implemented yet")
extern "C" {
pg_status pg_clustering(pg_ctx* ctx, const pg_graph*, int32_t, int32_t, float*, int64_t*, double*) { PENDING("pg_clustering"); }
pg_status pg_paths(pg_ctx* ctx, const pg_graph*, float*, double*, double*, int64_t*, int32_t, int32_t*) { PENDING("pg_paths"); }
pg_status pg_betweenness(pg_ctx* ctx, const pg_graph*, float*, double*, float*, double*) { PENDING("pg_betweenness"); }
pg_status pg_bfs_sigma(pg_ctx* ctx, const pg_graph*, const int32_t*, int32_t, int32_t*, int64_t*) { PENDING("pg_bfs_sigma"); }
pg_status pg_fw_paths(pg_ctx* ctx, const pg_graph*, float*, float*, double*) { PENDING("pg_fw_paths"); }
pg_status pg_fw_batched(pg_ctx* ctx, const pg_graph* const*, int32_t, float*, double*, float*, double*) { PENDING("pg_fw_batched"); }
pg_status pg_newman(pg_ctx* ctx, const pg_graph*, int32_t, int32_t*, double*, int32_t*, pg_log_fn, void*) { PENDING("pg_newman"); }
pg_status pg_maslov(pg_ctx* ctx, const pg_graph*, uint64_t, int64_t, pg_graph**, int64_t*) { PENDING("pg_maslov"); }
int64_t pg_maslov_round_size(int64_t M) { int64_t b = M / 16; if (b < 1) b = 1; if (b > 65536) b = 65536; return b; }
}
