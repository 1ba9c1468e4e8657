// elp_common.h -- pieces shared by the single-melt and batch C ABIs: error
// reporting, geometry choice, device-side ring reconstruction and checks,
// TUV text parsing.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/elp.h"
#include "elp_internal.h"

// Record a message for elp_last_error() and return `s`.
elp_status elp_fail(elp_status s, const char* fmt, ...);

#define ELP_CUDA_TRY(call)                                                                           \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return elp_fail(e_ == cudaErrorMemoryAllocation ? ELP_ERR_NOMEM : ELP_ERR_CUDA,          \
                            "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);    \
    } while (0)

// Rings and geometry of a job spec; returns ELP_OK or ELP_ERR_ARG.
elp_status elp_resolve_spec(const elp_job_spec* spec, int* P, elp_geometry* g);

// Device error flags written by kernels instead of trapping.
elp_status elp_device_errors(const uint32_t* d_flags, cudaStream_t s);

// Scratch buffers for walking rings on the device.
struct elp_walk_bufs {
    int32_t* d_start = nullptr;
    uint8_t* d_bonds = nullptr;
    int32_t* d_status = nullptr;
    uint32_t* d_visit = nullptr;
    unsigned long long* d_cnt = nullptr;
    unsigned long long* d_obs = nullptr;   // observables: [P][6] ring sums + histogram
    int32_t* h_status = nullptr;           // pinned host copies of the ring statuses and counters
    unsigned long long* h_cnt = nullptr;
    void* d_rank = nullptr;                // list ranking: 20 bytes a site (elp_rank.cu)
    uint32_t* d_total = nullptr;           // list ranking: monomers per chain
    size_t cap_rings = 0, cap_bonds = 0, cap_sites = 0, cap_obs = 0, cap_h_rings = 0, cap_rank_sites = 0, cap_total = 0;
    size_t bytes = 0;
};
void elp_walk_bufs_free(elp_walk_bufs* b);
// Grow the scratch to P chains of N and `sites` visit counters.
elp_status elp_walk_bufs_reserve(elp_walk_bufs* b, int P, int N, size_t sites);
// Build a melt's site words and chain records on the device from host chains
// (start[3*P], bonds[P*N]); ELP_ERR_INTEGRITY (codes 3/4) for invalid chains,
// which leave the lattice partly written.
elp_status elp_build_melt(uint32_t* lat, uint32_t* rec, int L, int N, int P, int linear, const int32_t* start,
                          const uint8_t* bonds, elp_walk_bufs* wb, cudaStream_t s);
// The reference initial melt (CreatePolymers) written on the device,
// stream-ordered: no transfer, no host wait.
elp_status elp_init_melt_device(uint32_t* lat, uint32_t* rec, int L, int N, int P, int linear, cudaStream_t s);

// Boxes up to this many sites (L = 512) rebuild their chains by list
// ranking; larger ones by the chain walk.
constexpr size_t ELP_RANK_MAX_SITES = (size_t)1 << 27;
// Chains of one melt into b->d_start / d_bonds / d_status by list ranking
// (elp_rank.cu), stream-ordered; cudaErrorNotSupported (nothing launched)
// above ELP_RANK_MAX_SITES sites.
cudaError_t elp_rank_chains(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear,
                            elp_walk_bufs* b, cudaStream_t s);
// Rebuild rings (start[3P], bonds[P*N]) of one melt into host buffers.
elp_status elp_fetch_rings(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                           int32_t* start, uint8_t* bonds, cudaStream_t s);
// Observables of one melt (elp_observe); any output may be null.
elp_status elp_observe_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                            double* cms_tuv, double* rg2, double* sl, uint64_t* run_hist, int nbins, cudaStream_t s);
// Rings of one melt into host buffers (pinned: the copies run behind the
// walk) together with its integrity code (0, 3 or 4), from one walk and one
// site scan.  A ring that cannot be walked gives code 4 with ELP_OK: the
// buffers are then unspecified.
elp_status elp_fetch_checked_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear,
                                  elp_walk_bufs* b, int32_t* start, uint8_t* bonds, int32_t* code, cudaStream_t s);
// Integrity check of one melt (code 0, 3 or 4 as CheckIntegrity).
elp_status elp_check_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                          int32_t* code, cudaStream_t s);

// Parse TUV text for a melt of box L, P rings of N.  Returns ELP_OK or
// ELP_ERR_FORMAT (message set).
elp_status elp_parse_tuv(const char* text, const char* name, int L, int N, int P, int32_t* start, uint8_t* bonds);
elp_status elp_read_file(const char* path, char** text, size_t* len);
