// bc_dense.cuh -- forward Brandes levels as exact integer GEMMs on the tensor
// cores (tcgen05 kind::i8), for graphs whose dense 0/1 adjacency fits the
// device.  Used by brandes.cu for the levels where most (node, source) pairs
// are active.
#pragma once
#include "pg_internal.cuh"
#include <cuda.h>

struct BCDense {
    int n = 0;                   // nodes
    int np = 0;                  // nodes padded to 128
    int max_deg = 0;
    uint8_t* adj = nullptr;      // np x np, adj[v * np + u] = 1 for an edge
    uint8_t* xt = nullptr;       // limbs (<= 2) x 128 x np: level-(d-1) path counts, transposed
    int* err = nullptr;          // set when a pipeline wait timed out
    int32_t* tail = nullptr;     // partial sums of the K-split tail tiles
    CUtensorMap map_adj;
};

// State of one 128-source batch (layout of brandes.cu: [node][128 sources]).
struct BCLevel {
    unsigned long long* sigma;   // [n][128]
    int32_t* dist;               // [n][128]
    ulonglong2* seen;            // [n] sources that reached the node
    ulonglong2* nxt;             // [n] frontier written for level d
    const ulonglong2* fprev;     // [n] frontier of level d - 1
    ulonglong2* fhist;           // [n] frontier history slot of level d (null: none)
    double* inv;                 // [n] sum of 1/d (null: skip)
    int* flag;                   // set to 1 when level d reaches a node
    int d;                       // level
};

// Dense levels pay off when the adjacency fits in a bounded share of the
// device memory and rows are long (a pass over the dense matrix costs what a
// gather pass over about np^2 / 64 edges does).
bool bc_dense_eligible(pg_ctx* ctx, int n, long long nnz, int max_deg);
pg_status bc_dense_setup(pg_ctx* ctx, const int32_t* R, const int32_t* C, int n, BCDense& d);
// Level d from level d - 1: sigma_d[v][s] = sum_u adj[v][u] sigma_{d-1}[u][s]
// over the u on level d - 1 of source s, kept where v was not yet reached.
pg_status bc_dense_level(pg_ctx* ctx, BCDense& d, const BCLevel& lv);
// Fails if any dense level of this setup timed out (synchronises the stream).
pg_status bc_dense_check(pg_ctx* ctx, BCDense& d);
