// elp_rank.cu -- chain reconstruction by list ranking (pointer jumping).
//
// The chains of a melt are linked lists through the site words: a run's
// b_out leads to the next run's site.  walk_kernel (elp_walk.cu) follows
// each chain run by run, a chain of several hundred dependent loads per ring
// of a relaxed melt, so its time is one ring's latency.  Here every run
// takes part at once: after cutting each list in front of its labelled run
// (the run holding monomer 0), every site jumps along its list by doubling
// strides (Wyllie's list ranking), ceil(log2 N) rounds over the lattice, and
// learns the monomers from its run to the chain's last run and which run
// that is.  The chain's labelled run then knows the chain's length and its
// last run; every run knows its monomers' place in its chain and writes its
// bond.  The output is the TUV content of cpupol/efpol_io.c:70-77 (start
// site of monomer 0, N bond codes), the same bytes as walk_kernel writes,
// and a chain that walk_kernel would reject (a bond that is not a lattice
// bond, a run leading to an empty site or into another chain, a wrong
// monomer count) gets status 4 here too; so does a chain with runs joined to
// it from outside (counted per chain).
#include <cuda_runtime.h>

#include "elp_common.h"
#include "elp_internal.h"

namespace elp {
namespace {

// Per-site state {link, sum}.  link < FIN: a later site of the same chain,
// sum the monomers from this run up to that site's run (exclusive).  link
// with FIN set: finished, the low bits name the chain's last run (its tail)
// and sum counts the monomers from this run to the tail (inclusive).  EMPTY:
// no run on the site.
constexpr uint32_t FIN = 0x80000000u;
constexpr uint32_t EMPTY = 0xFFFFFFFFu;

struct RankArgs {
    const uint32_t* lat;
    const uint32_t* rec;
    int L, N, P, linear;
    uint2* x[2];                // double-buffered per-site state
    int32_t* chain_of_tail;     // per site: the chain whose last run it is, else -1
    uint32_t* total;            // per chain: monomers of the runs that reached its tail
    int32_t* start;             // [P][3]
    uint8_t* bonds;             // [P][N], zeroed before
    int32_t* status;            // [P]
};

__device__ __forceinline__ uint32_t step_site(uint32_t s, uint32_t b, int L)
{
    const uint32_t uL = (uint32_t)L;
    int t = (int)(s % uL), u = (int)((s / uL) % uL), v = (int)(s / (uL * uL));
    t += elp_bt(b); u += elp_bu(b); v += elp_bv(b);
    t += t < 0 ? L : 0; t -= t >= L ? L : 0;
    u += u < 0 ? L : 0; u -= u >= L ? L : 0;
    v += v < 0 ? L : 0; v -= v >= L ? L : 0;
    return (uint32_t)t + uL * ((uint32_t)u + uL * (uint32_t)v);
}

// Monomers of the run on a site, counted from monomer 0 for the labelled
// run (those ahead of monomer 0 close the ring); 0 for a label naming no
// valid chain record (the chain check rejects it).
__device__ __forceinline__ uint32_t run_weight(uint32_t w, const RankArgs& a)
{
    if (!(w & ELP_LBIT)) return w >> ELP_CSHIFT;
    const uint32_t ch = w >> 5;
    if (ch >= (uint32_t)a.P) return 0;
    const uint32_t cnt = a.rec[ELP_REC_WORDS * (size_t)ch + 1], off = a.rec[ELP_REC_WORDS * (size_t)ch + 2];
    return off < cnt ? cnt - off : 0;
}

__global__ void rank_init(RankArgs a)
{
    const uint32_t S = (uint32_t)a.L * a.L * a.L;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const uint32_t w = a.lat[s];
        if (!w) {
            a.x[0][s] = a.x[1][s] = make_uint2(EMPTY, 0u);
            continue;
        }
        // a run is its chain's last unless a plain (unlabelled) run follows:
        // the lists are cut in front of every labelled run
        uint32_t link = FIN | s;
        const uint32_t bo = w & 15;
        if (elp_valid_bond(bo)) {
            const uint32_t n = step_site(s, bo, a.L);
            const uint32_t wn = a.lat[n];
            if (wn && !(wn & ELP_LBIT)) link = n;
        }
        a.x[0][s] = make_uint2(link, run_weight(w, a));
    }
}

// One doubling round: every unfinished site adds its successor's sum and
// takes its successor's link.
__global__ void rank_round(RankArgs a, int r)
{
    const uint32_t S = (uint32_t)a.L * a.L * a.L;
    const uint2* in = a.x[r & 1];
    uint2* out = a.x[(r & 1) ^ 1];
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        uint2 e = in[s];
        if (e.x == EMPTY) continue;
        if (!(e.x & FIN)) {
            const uint2 f = in[e.x];
            e = make_uint2(f.x, e.y + f.y);
        }
        out[s] = e;
    }
}

// Per chain: its labelled run must have reached the chain's tail with the
// chain's monomer count, and the tail must close the ring on the labelled
// run (a linear chain: end in the marker 0xf).
__global__ void rank_chains(RankArgs a, int fin)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.P) return;
    const uint32_t S = (uint32_t)a.L * a.L * a.L;
    const uint32_t site = a.rec[ELP_REC_WORDS * (size_t)p], cnt = a.rec[ELP_REC_WORDS * (size_t)p + 1],
                   off = a.rec[ELP_REC_WORDS * (size_t)p + 2];
    bool bad = site >= S || cnt == 0 || off >= cnt || (a.linear && off != 0);
    if (!bad) {
        const uint32_t w = a.lat[site];
        bad = !(w & ELP_LBIT) || (w >> 5) != (uint32_t)p;
    }
    uint32_t tail = 0;
    if (!bad) {
        const uint2 e = a.x[fin][site];
        const uint32_t expect = a.linear ? (uint32_t)a.N : (uint32_t)a.N - off;
        bad = e.x == EMPTY || !(e.x & FIN) || e.y != expect;
        tail = e.x & ~FIN;
    }
    if (!bad) {
        const uint32_t bo = a.lat[tail] & 15;
        bad = a.linear ? bo != 15 : (!elp_valid_bond(bo) || step_site(tail, bo, a.L) != site);
    }
    if (!bad) {
        a.chain_of_tail[tail] = p;
        const uint32_t uL = (uint32_t)a.L;
        a.start[3 * p] = (int32_t)(site % uL);
        a.start[3 * p + 1] = (int32_t)((site / uL) % uL);
        a.start[3 * p + 2] = (int32_t)(site / (uL * uL));
    }
    a.status[p] = bad ? 4 : 0;
}

// Per run of a good chain: the bond of its last monomer, at that monomer's
// place in the chain (the other monomers of a run are stored: bond 0).
__global__ void rank_bonds(RankArgs a, int fin)
{
    const uint32_t S = (uint32_t)a.L * a.L * a.L;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const uint2 e = a.x[fin][s];
        if (e.x == EMPTY || !(e.x & FIN)) continue;
        const int p = a.chain_of_tail[e.x & ~FIN];
        if (p < 0) continue;
        const uint32_t w = a.lat[s];
        const uint32_t weight = run_weight(w, a);
        const uint32_t off = a.linear ? 0u : a.rec[ELP_REC_WORDS * (size_t)p + 2];
        const long idx = (long)a.N - (long)off - (long)e.y + (long)weight - 1;
        if (weight == 0 || idx < 0 || idx >= (long)a.N) {
            atomicExch(&a.status[p], 4);
            continue;
        }
        a.bonds[(size_t)p * a.N + (size_t)idx] = (uint8_t)(w & 15);
        atomicAdd(&a.total[p], weight);
    }
}

// A chain whose tail was also reached by runs off its path holds more
// monomers than the path from its labelled run: rejected.
__global__ void rank_totals(RankArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.P || a.status[p]) return;
    const uint32_t off = a.linear ? 0u : a.rec[ELP_REC_WORDS * (size_t)p + 2];
    if (a.total[p] != (uint32_t)a.N - off) a.status[p] = 4;
}

}  // namespace
}  // namespace elp

// Chains of one melt into d_start / d_bonds / d_status (device scratch of
// b), stream-ordered; the caller copies them out.  Sites beyond
// ELP_RANK_MAX_SITES are not ranked (the scratch would be 20 bytes a site):
// returns cudaErrorNotSupported without launching anything.
cudaError_t elp_rank_chains(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear,
                            elp_walk_bufs* b, cudaStream_t s)
{
    const size_t S = (size_t)L * L * L;
    if (S > ELP_RANK_MAX_SITES || P <= 0) return cudaErrorNotSupported;
    cudaError_t e;
    if (S > b->cap_rank_sites) {
        cudaFree(b->d_rank);
        b->d_rank = nullptr;
        b->bytes -= b->cap_rank_sites * 20;
        b->cap_rank_sites = 0;
        if ((e = cudaMalloc(&b->d_rank, S * 20)) != cudaSuccess) return e;
        b->cap_rank_sites = S;
        b->bytes += S * 20;
    }
    if ((size_t)P > b->cap_total) {
        cudaFree(b->d_total);
        b->d_total = nullptr;
        b->bytes -= b->cap_total * 4;
        b->cap_total = 0;
        if ((e = cudaMalloc((void**)&b->d_total, (size_t)P * 4)) != cudaSuccess) return e;
        b->cap_total = (size_t)P;
        b->bytes += (size_t)P * 4;
    }
    elp::RankArgs a;
    a.lat = lat; a.rec = rec; a.L = L; a.N = N; a.P = P; a.linear = linear;
    a.x[0] = reinterpret_cast<uint2*>(b->d_rank);
    a.x[1] = a.x[0] + S;
    a.chain_of_tail = reinterpret_cast<int32_t*>(a.x[1] + S);
    a.total = b->d_total;
    a.start = b->d_start; a.bonds = b->d_bonds; a.status = b->d_status;
    if ((e = cudaMemsetAsync(a.chain_of_tail, 0xFF, S * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.total, 0, (size_t)P * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.bonds, 0, (size_t)P * N, s)) != cudaSuccess) return e;
    int blocks = (int)((S + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    // a chain has at most N runs: 2^R >= N strides reach its tail from any run
    int R = 0;
    while ((1L << R) < (long)N) R++;
    elp::rank_init<<<blocks, 256, 0, s>>>(a);
    for (int r = 0; r < R; r++) elp::rank_round<<<blocks, 256, 0, s>>>(a, r);
    const int fin = R & 1;
    const int cb = (P + 255) / 256;
    elp::rank_chains<<<cb, 256, 0, s>>>(a, fin);
    elp::rank_bonds<<<blocks, 256, 0, s>>>(a, fin);
    elp::rank_totals<<<cb, 256, 0, s>>>(a);
    return cudaGetLastError();
}
