// elp_noalloc.cu -- integrity check that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: an application that
// has handed the whole device memory to its own pool, a process running under
// a device-memory quota, or a latency-critical loop that cannot take the
// implicit device synchronisation and unbounded time of an allocation.  For
// them elp_check_noalloc runs the same walk and scan kernels as elp_check,
// but its scratch memory (one visit counter per site, one status per ring,
// eight counters) is a fixed array in this file's device memory, loaded with
// the library on every GPU that uses it and held until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the parts that must start at zero are cleared on the caller's
// stream before the kernels run.  Calls that overlap on the GPU (two streams,
// or two threads) race on the array and must be serialised by the caller.
// The walk follows rings: a melt of linear chains gets code 4.  The array's
// device address is looked up once per device and kept; after a device reset
// (cudaDeviceReset) the module can come back at another address, so a
// process that resets a device must not call this entry point again.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "elp_common.h"
#include "elp_kernels.h"

namespace {
struct NoAllocScratch {
    uint32_t visit[ELP_NOALLOC_MAX_SITES];
    int32_t status[ELP_NOALLOC_MAX_RINGS];
    unsigned long long counters[8];
};
}  // namespace

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Host code may not use g_noalloc_scratch as an address: on the host the
// name stands for a host-side shadow.  The device address comes from
// cudaGetSymbolAddress, once per device, with that device current.
static std::mutex g_noalloc_mu;
static NoAllocScratch* g_noalloc_addr[128];

__global__ void noalloc_bad_rings_kernel(const int32_t* status, int P, unsigned long long* counters)
{
    unsigned long long bad = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) bad += status[p] != 0;
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&counters[6], bad);
}

extern "C" elp_status elp_check_noalloc(const uint32_t* d_words, const uint32_t* d_records, int32_t L, int32_t N,
                                        int32_t P, void* stream, int32_t* code)
{
    if (!d_words || !d_records || !code) return elp_fail(ELP_ERR_ARG, "null argument");
    if (L < 5 || N < 3 || P < 1) return elp_fail(ELP_ERR_ARG, "bad melt size L=%d N=%d P=%d", L, N, P);
    const size_t S = (size_t)L * L * L;
    if (S > ELP_NOALLOC_MAX_SITES)
        return elp_fail(ELP_ERR_ARG, "elp_check_noalloc handles at most %u sites (L <= 64); L=%d has %zu",
                        (unsigned)ELP_NOALLOC_MAX_SITES, L, S);
    if ((size_t)P > ELP_NOALLOC_MAX_RINGS)
        return elp_fail(ELP_ERR_ARG, "elp_check_noalloc handles at most %u rings; got %d",
                        (unsigned)ELP_NOALLOC_MAX_RINGS, P);
    int dev = 0;
    ELP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return elp_fail(ELP_ERR_ARG, "device ordinal %d out of range", dev);
    NoAllocScratch* sc;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return elp_fail(ELP_ERR_CUDA, "cannot locate the static scratch array on device %d: %s", dev,
                                cudaGetErrorString(e));
            g_noalloc_addr[dev] = static_cast<NoAllocScratch*>(ptr);
        }
        sc = g_noalloc_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ELP_CUDA_TRY(cudaMemsetAsync(sc->visit, 0, S * sizeof(uint32_t), s));
    ELP_CUDA_TRY(cudaMemsetAsync(sc->counters, 0, sizeof(sc->counters), s));
    WalkArgs w;
    memset(&w, 0, sizeof(w));
    w.lat = d_words;
    w.rec = d_records;
    w.L = L;
    w.N = N;
    w.P = P;
    w.status = sc->status;    // every ring p < P gets a status
    w.visit = sc->visit;
    w.counters = sc->counters;
    ELP_CUDA_TRY(elp_launch_walk(&w, s));
    ELP_CUDA_TRY(elp_launch_scan(&w, s));
    int blocks = (P + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    noalloc_bad_rings_kernel<<<blocks, 256, 0, s>>>(sc->status, P, sc->counters);
    ELP_CUDA_TRY(cudaGetLastError());
    unsigned long long cnt[8];
    ELP_CUDA_TRY(cudaMemcpyAsync(cnt, sc->counters, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    int rc = 0;
    if (cnt[6]) rc = 4;
    if (!rc && cnt[4]) rc = 3;
    if (!rc && (cnt[0] != cnt[1] || cnt[2] != (unsigned long long)N * P || cnt[3])) rc = 4;
    *code = rc;
    return ELP_OK;
}
