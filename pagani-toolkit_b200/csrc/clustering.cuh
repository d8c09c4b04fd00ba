// clustering.cuh -- clustering pieces that the surrogate pipeline (runner.cu)
// and the batched FW tool enqueue without host round trips.
#pragma once
#include "pg_internal.cuh"

struct BinaryCpArgs {
    unsigned long long* tri2;   // per node: twice the triangle count
    int* counter;               // dynamic node scheduler
    size_t smem;                // neighbour bitmap bytes
};
// Sizes the workspace and sets the kernel's shared-memory limit.
pg_status binary_cp_prepare(pg_ctx* ctx, int n, BinaryCpArgs* a);
// Enqueues Cp (U/Cp/Cp/Cp.cpp:21-116) of (R, C): cp float[n], exact
// triangles (tri, optional), FP64 mean over all n nodes -- device pointers.
pg_status binary_cp_enqueue(pg_ctx* ctx, const BinaryCpArgs* a, const int32_t* R, const int32_t* C, int n, float* cp,
                            long long* tri, double* mean);

struct OnnelaArgs {
    void* tab;                  // device table of graphs
    int* node0;
    int* counter;
    float* vmax;
    size_t smem;
    int ng, total, first_n;
    float* cp;
    double* mean;
};
// Uploads the table of graphs (synchronises the stream); the graphs' device
// arrays must stay where they are while the arguments are used.
pg_status onnela_prepare(pg_ctx* ctx, const pg_graph* const* graphs, int ng, int first_n, float* cp_dev,
                         double* mean_dev, OnnelaArgs* a);
// Enqueues Onnela clustering (W/Cp/Cp/Cp_2.cpp:23-130) of every graph of the table.
pg_status onnela_enqueue(pg_ctx* ctx, const OnnelaArgs* a);
