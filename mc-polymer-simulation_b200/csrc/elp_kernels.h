// elp_kernels.h -- launch interfaces of the device kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct SweepArgs {
    uint32_t* lat;                 // L^3 site words
    uint32_t* rec;                 // chain records
    const uint32_t* table;         // 1024 words = 4096 bytes dst1|dst2<<4
    unsigned long long* accepted;  // optional accepted-move counter
    uint32_t* error;               // device error flags (bit 0: label slot table overflow,
                                   // bit 2: a dependency wait gave up)
    int nchains;                   // rings in the melt
    int L, periodic, tx, ty, tz, ncol;
    int sx, sxy, ox, words, groups;
    uint32_t seed, salt;
    uint64_t step0;
    int nsteps;
};

struct WalkArgs {
    const uint32_t* lat;
    const uint32_t* rec;
    int L, N, P;
    int32_t* start;                // [P][3] or null
    uint8_t* bonds;                // [P][N] or null
    int32_t* status;               // [P]
    uint32_t* visit;               // [L^3] visit counters or null
    unsigned long long* counters;  // [5]: runs walked, runs found, monomers found, bad sites, shared sites
    int linear;                    // 1: chains end in a run with b_out 0xf instead of closing
};

// One melt of a batch as the specialised kernel sees it.
struct BatchJob {
    uint32_t* lat;                 // its L^3 site words
    uint32_t* rec;                 // its chain records
    unsigned long long* acc;       // its accepted-move counter (or null)
    int L, nchains;
    int ntx, nty, ntz;             // domains per axis
    uint32_t seed, salt;
    uint32_t step0;                // absolute step at step_base == 0
    int linear;                    // 1: linear chains (head moves of monomer 0 at its anchor)
};

struct BatchLaunch {
    const BatchJob* jobs;          // device job table
    const uint2* items;            // device work items {job, domain}
    int nitems;
    int nsteps;                    // steps per launch
    uint32_t step_base;            // added to every job's step0 ...
    const uint32_t* step_dev;      // ... and, if set, this device counter (graph replays)
    const uint32_t* table;         // 4096-byte transition table
    uint32_t* error;               // device error flags (bit 0: label slot table overflow,
                                   // bit 2: a grid barrier wait gave up)
    uint32_t* grid_bar;            // tiled domains, nsteps > 1: {arrivals, exits}, zero between launches
    uint32_t wait_polls;           // polls before a grid barrier wait gives up (0: about a second)
    int hold_cta1;                 // test hook: CTA + 1 that never arrives at the first barrier (0: none)
};

#include "elp_internal.h"
struct Sweep2Launch {
    elp_geometry geom;
    int sx, sxy;                   // shared-memory strides of the layout
    int nsm;                       // SMs for the persistent grid
    int check_only;                // only report whether a kernel fits
    double max_runs_per_domain;    // expected monomer-0 runs in one domain
    BatchLaunch args;
    int threads_out;               // check_only: block size of the kernel that fits
    size_t smem_out;               // check_only: its dynamic shared memory
    int linear;                    // 1: some job holds linear chains (kernel with monomer-0 moves)
};

extern "C" {
cudaError_t elp_launch_sweep(const SweepArgs* a, int ndomains, int threads, size_t smem, cudaStream_t s);
cudaError_t elp_launch_sweep2(const Sweep2Launch* l, cudaStream_t s);
cudaError_t elp_launch_walk(const WalkArgs* a, cudaStream_t s);
cudaError_t elp_launch_scan(const WalkArgs* a, cudaStream_t s);
}
