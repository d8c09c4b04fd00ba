// gram_tc.cu -- split-BF16 Gram on the tcgen05 tensor cores (placeholder
// until the TMEM kernel lands; reports the path as unsupported).
#include "build_graph.cuh"

bool gram_tc_supported(pg_ctx*, const ZOperands&) { return false; }

pg_status launch_gram_tc(pg_ctx* ctx, const ZOperands&, int, const EpiParams&)
{
    return pg_fail(ctx, PG_ERR_INVALID, "tcgen05 Gram not available");
}
