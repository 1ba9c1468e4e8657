// elp_walk.cu -- chain reconstruction and invariant kernels.
//
// walk_kernel rebuilds each ring (start site of monomer 0 plus N bond codes,
// the TUV content of cpupol/efpol_io.c:70-77) from the site words by
// following b_out from monomer 0's run; it replaces the reference's host-side
// GetAllRingPolymers / UpdatePolymerWithLabels (gpupol2/oclpol.c:183-376).
// With visit counters it also proves the integrity conditions of the
// reference's CheckIntegrity (cpupol/efpol_io.c:158-211): every ring closes
// after exactly N monomers through valid bonds (a linear chain instead ends
// after exactly N monomers in a run whose b_out is the marker 0xf, with
// monomer 0 first in its run), and (with scan_kernel) every occupied site
// belongs to exactly one chain and the monomer total is N*P.
#include <cuda_runtime.h>

#include "elp_internal.h"
#include "elp_kernels.h"

namespace elp {

__device__ __forceinline__ uint32_t step_site(uint32_t cur, uint32_t b, int L)
{
    int t = (int)(cur % (uint32_t)L), u = (int)((cur / (uint32_t)L) % (uint32_t)L), v = (int)(cur / ((uint32_t)L * L));
    t += elp_bt(b); u += elp_bu(b); v += elp_bv(b);
    t += t < 0 ? L : 0; t -= t >= L ? L : 0;
    u += u < 0 ? L : 0; u -= u >= L ? L : 0;
    v += v < 0 ? L : 0; v -= v >= L ? L : 0;
    return (uint32_t)t + (uint32_t)L * ((uint32_t)u + (uint32_t)L * (uint32_t)v);
}

__global__ void walk_kernel(WalkArgs a)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.P) return;
    const int L = a.L, N = a.N;
    const size_t S = (size_t)L * L * L;
    uint32_t site = a.rec[ELP_REC_WORDS * p], cnt = a.rec[ELP_REC_WORDS * p + 1], off = a.rec[ELP_REC_WORDS * p + 2];
    int bad = 0;
    if (site >= S || off >= cnt || cnt == 0 || (a.linear && off != 0)) bad = 1;
    uint32_t w = bad ? 0 : a.lat[site];
    if (!bad && (!(w & ELP_LBIT) || (w >> 5) != (uint32_t)p)) bad = 1;
    if (bad) { a.status[p] = 4; return; }
    if (a.start) {
        a.start[3 * p] = (int32_t)(site % (uint32_t)L);
        a.start[3 * p + 1] = (int32_t)((site / (uint32_t)L) % (uint32_t)L);
        a.start[3 * p + 2] = (int32_t)(site / ((uint32_t)L * L));
    }
    uint8_t* b = a.bonds ? a.bonds + (size_t)p * N : nullptr;
    long i = 0;
    uint32_t here = cnt - off, cur = site;
    unsigned long long runs = 0;
    for (;;) {
        uint32_t bo = a.lat[cur] & 15;
        const bool end = a.linear && bo == 15;   // last run of a linear chain
        if (!(elp_valid_bond(bo) || end) || i + (long)here > (long)N) { bad = 1; break; }
        if (b) {
            for (uint32_t k = 0; k + 1 < here; k++) b[i + k] = 0;
            b[i + here - 1] = (uint8_t)bo;
        }
        i += here;
        runs++;
        if (a.visit) atomicAdd(&a.visit[cur], 1u);
        if (end) break;
        cur = step_site(cur, bo, L);
        uint32_t wn = a.lat[cur];
        if (!wn) { bad = 1; break; }
        if (cur == site) break;
        if (wn & ELP_LBIT) { bad = 1; break; }
        here = wn >> ELP_CSHIFT;
        if (here == 0 || runs >= (unsigned long long)N) { bad = 1; break; }
    }
    if (!bad && i + (long)off != N) bad = 1;
    if (!bad && b)
        for (uint32_t k = 0; k < off; k++) b[i + k] = 0;
    a.status[p] = bad ? 4 : 0;
    if (a.counters) atomicAdd(&a.counters[0], runs);
}

__global__ void scan_kernel(WalkArgs a)
{
    const size_t S = (size_t)a.L * a.L * a.L;
    unsigned long long runs = 0, mono = 0, badc = 0, multi = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < S; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t w = a.lat[i];
        uint32_t v = a.visit ? a.visit[i] : 0;
        if (!w) {
            if (v) badc++;
            continue;
        }
        runs++;
        uint32_t c;
        if (w & ELP_LBIT) {
            uint32_t ch = w >> 5;
            if (ch >= (uint32_t)a.P || a.rec[ELP_REC_WORDS * ch] != (uint32_t)i) { badc++; continue; }
            c = a.rec[ELP_REC_WORDS * ch + 1];
        } else {
            c = w >> ELP_CSHIFT;
            if (w & 0xFFE0u) badc++;   // bits 5-15 must be clear
        }
        mono += c;
        if (!(elp_valid_bond(w & 15) || (a.linear && (w & 15) == 15)) || c == 0 || (a.visit && v == 0)) badc++;
        if (a.visit && v > 1) multi++;
    }
    for (int o = 16; o > 0; o >>= 1) {
        runs += __shfl_xor_sync(0xffffffffu, runs, o);
        mono += __shfl_xor_sync(0xffffffffu, mono, o);
        badc += __shfl_xor_sync(0xffffffffu, badc, o);
        multi += __shfl_xor_sync(0xffffffffu, multi, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&a.counters[1], runs);
        atomicAdd(&a.counters[2], mono);
        atomicAdd(&a.counters[3], badc);
        atomicAdd(&a.counters[4], multi);
    }
}

}  // namespace elp

extern "C" cudaError_t elp_launch_walk(const WalkArgs* a, cudaStream_t s)
{
    if (a->P <= 0) return cudaSuccess;
    elp::walk_kernel<<<(a->P + 127) / 128, 128, 0, s>>>(*a);
    return cudaGetLastError();
}

extern "C" cudaError_t elp_launch_scan(const WalkArgs* a, cudaStream_t s)
{
    size_t S = (size_t)a->L * a->L * a->L;
    int blocks = (int)((S + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    elp::scan_kernel<<<blocks, 256, 0, s>>>(*a);
    return cudaGetLastError();
}
