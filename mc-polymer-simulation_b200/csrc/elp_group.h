// elp_group.h -- melts that share one domain geometry and advance together.
//
// A group owns a device job table (one BatchJob per melt), the work items
// {melt, domain} of a step, a device step counter and a stream.  Both the
// single-melt context (a group of one) and the batch API are built on it, so
// a melt run alone and the same melt run inside a batch execute the same
// kernel with the same counters and give the same bits.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "elp_internal.h"
#include "elp_kernels.h"

struct elp_group {
    elp_geometry g;
    elp_smem_layout lay;
    int nsm;
    int generic;                      // force the generic kernel
    int specialised;                  // a specialised kernel fits this group
    int threads;                      // block size of the sweep kernel in use
    size_t smem;                      // its dynamic shared memory per block
    int spl;                          // steps per launch (tiled: specialised kernel only)
    int use_graph;                    // tiled domains: replay launches from a CUDA graph
    int graph_steps;                  // steps captured per graph (rounded down to whole launches)
    cudaStream_t stream;
    const uint32_t* d_table;
    uint32_t* d_error;

    std::vector<BatchJob> jobs;       // host mirror of the job table
    std::vector<int> N;               // ring length per melt
    BatchJob* d_jobs = nullptr;
    uint2* d_items = nullptr;
    int nitems = 0;
    size_t cap_jobs = 0, cap_items = 0;   // grow-only device capacity of the two tables
    uint32_t* d_ctr = nullptr;        // device step counter, then the grid barrier's two counts
    uint32_t wait_polls = 0;          // bound of the grid barrier's waits (0: the kernel's default)
    int hold_cta1 = 0;                // test hook: CTA + 1 that never arrives at the first barrier
    uint64_t steps_done = 0;          // steps since the job table's step0 values
    uint32_t ctr_mirror = 0;          // host copy of *d_ctr
    uint64_t kernels = 0;             // sweep-path kernels launched (graph replays count their nodes)

    cudaGraphExec_t graph = nullptr;
    uint32_t graph_base = 0;          // step_base offset the graph was captured with
};

// Set up a group for `geom`; melts are added with elp_group_add.
cudaError_t elp_group_init(elp_group* G, const elp_geometry& geom, int nsm, int generic, int spl,
                           const uint32_t* d_table, uint32_t* d_error, cudaStream_t stream);
void elp_group_add(elp_group* G, uint32_t* lat, uint32_t* rec, unsigned long long* acc, int N, int nchains,
                   uint32_t seed, uint32_t salt, uint64_t step, int linear);
// Upload the job table and work items; decide specialised vs generic.
cudaError_t elp_group_commit(elp_group* G);
// Set the absolute step of melt j (after loading a configuration).
cudaError_t elp_group_set_step(elp_group* G, int j, uint64_t step);
uint64_t elp_group_step(const elp_group* G, int j);
// Enqueue nsteps steps of every melt in the group on its stream.
cudaError_t elp_group_run(elp_group* G, int64_t nsteps);
void elp_group_free(elp_group* G);
