// maslov.cuh -- the Maslov rewiring pieces that the surrogate pipeline
// (runner.cu) enqueues without host round trips.
#pragma once
#include "pg_internal.cuh"

// Round counters of one rewiring, in device memory.
struct MsControl {
    unsigned long long n_pending[2];  // deferred attempts carried into a round (by round parity)
    unsigned long long oldest[2];     // smallest index among them
    unsigned long long committed;
    unsigned long long rounds;
};

struct MsArgs {
    int n;
    long long M;                     // undirected edges (slots)
    long long B;                     // attempts per round
    uint32_t hmask;                  // pair table size - 1
    uint64_t seed;
    uint64_t attempts;
    size_t words;                    // edge bitmap words
    int grid;                        // cooperative grid of k_ms_rounds
    int32_t* cnt;
    long long* off;
    int *ea, *eb;                    // slot end points
    float* ew;                       // slot weights
    unsigned long long* bits;        // edge bitmap over the n(n-1)/2 unordered pairs
    // claims and write records: round tag << 32 | attempt index relative to
    // the round's oldest (lowest wins)
    unsigned long long* slot_owner;  // per slot: lowest claiming attempt
    unsigned long long* table;       // per pair entry: lowest claiming attempt
    unsigned long long* pair_wr;     // per pair entry: lowest committed attempt removing that pair
    void* items;                     // per round item: the evaluated attempt
    unsigned long long *pend_a, *pend_b;
    MsControl* st;
    const uint64_t* seed_dev;        // optional: seed = seed_dev[*round_dev] (one captured graph, many seeds)
    const int* round_dev;
    int32_t* cursor;                 // row cursors of the rebuild
    int32_t* ct;                     // unsorted rows of the rebuild
    float* vt;
};

// Round size and pair-table size for M slots (fixed functions of M, so the
// surrogate of a seed does not depend on anything else).
int64_t ms_round_size(int64_t M);
uint32_t ms_table_size(int64_t B);
// Sizes the workspace (may allocate) and fills the arguments.
pg_status ms_prepare(pg_ctx* ctx, const pg_graph* g, uint64_t seed, int64_t attempts, MsArgs* a);
// Enqueues the rewiring of g on the context stream: result slots in
// a->ea / a->eb (and a->ew); no allocation, no host synchronisation.
pg_status ms_enqueue(pg_ctx* ctx, const pg_graph* g, MsArgs* a);
// Enqueues the rows of the rewired graph: R is g->R (unchanged), columns
// ascending into C_out (nnz entries), weights into V_out (null: binary).
pg_status ms_rows_enqueue(pg_ctx* ctx, const pg_graph* g, MsArgs* a, int32_t* C_out, float* V_out);
