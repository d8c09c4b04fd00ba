// paths.cuh -- hop path length pieces that the surrogate pipeline
// (runner.cu) enqueues without host round trips.
#pragma once
#include "pg_internal.cuh"

constexpr int MAX_D = 64;   // per-node distance counters kept exactly; farther distances summed directly

struct PathArgs {
    int n;
    const int32_t* R;
    const int32_t* C;
    int nw;                    // 64-bit source words per node (4: 256 sources per batch, 8: 512)
    int ctas_per_sm;
    int max_hop;
    void *front, *next, *seen_a, *seen_b;   // per-node source bit words
    unsigned* cnt;             // n x MAX_D: sources reached at distance d
    double* inv_far;           // sum of 1/d over distances > MAX_D
    double* inv;               // sum_s 1/d(s, v)
    float* eff;                // inv / (n - 1)
    unsigned long long* hist;  // ordered pairs per distance (d <= max_hop)
    int* flags;                // "a source grew at level d" (three, rotating)
    int* diameter;
    double* out;               // [0] sum of inv, [1] Lp = n(n-1) / sum
};

// Sizes the workspace (may allocate) and picks the launch shape (autotuned).
pg_status paths_prepare(pg_ctx* ctx, const pg_graph* g, int max_hop, PathArgs* a);
// Enqueues the whole computation on the context stream: no allocation, no
// host synchronisation.
pg_status paths_enqueue(pg_ctx* ctx, PathArgs* a);
