// elp_kernels.h -- launch interfaces of the device kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct SweepArgs {
    uint32_t* lat;                 // L^3 site words
    uint32_t* rec;                 // chain records
    const uint32_t* table;         // 1024 words = 4096 bytes dst1|dst2<<4
    unsigned long long* accepted;  // optional accepted-move counter
    uint32_t* error;               // device error flags (bit 0: label slot table overflow)
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
};

extern "C" {
cudaError_t elp_launch_sweep(const SweepArgs* a, int ndomains, int threads, size_t smem, cudaStream_t s);
cudaError_t elp_launch_sweep2(const SweepArgs* a, int nsm, cudaStream_t s);
cudaError_t elp_launch_walk(const WalkArgs* a, cudaStream_t s);
cudaError_t elp_launch_scan(const WalkArgs* a, cudaStream_t s);
}
