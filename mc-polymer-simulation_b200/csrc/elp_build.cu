// elp_build.cu -- site words and chain records built on the device from
// chains (start site of monomer 0 plus N bond codes per chain, the content
// of a TUV file, cpupol/efpol_io.c:3-47).
//
// The load path ships only the chains to the device (12 P + N P bytes) and
// builds the lattice there, instead of building L^3 site words on the host
// and copying them.  build_kernel (one warp per chain) checks the bonds
// (valid codes; a ring closes, a linear chain ends in the marker 0xf), finds
// the chain's runs and claims each run's site with a compare-and-swap on the
// zeroed lattice: a site claimed twice means two runs on one site, efpol's
// CheckIntegrity code 3 (cpupol/efpol_io.c:182-187); a bad bond or an open
// ring is code 4.
#include <cuda_runtime.h>
#include <limits.h>

#include <vector>

#include "elp_common.h"
#include "elp_internal.h"

namespace elp {

struct BuildArgs {
    const int32_t* start;   // [P][3]
    const uint8_t* bonds;   // [P][N]
    uint32_t* lat;          // [L^3], zeroed
    uint32_t* rec;          // [P][4]
    int32_t* status;        // [P]: 0, 3 or 4
    int L, N, P, linear;
};

__device__ __forceinline__ int wrap(int x, int L)
{
    x %= L;
    return x < 0 ? x + L : x;
}

// One warp per chain.  Lane l owns monomers [l C, (l+1) C), C = ceil(N/32):
// a warp prefix sum of the bond vectors gives each lane the position of its
// first monomer, a suffix minimum gives the first non-zero bond after its
// chunk (where a run that leaves the chunk ends), and each lane then claims
// the sites of the runs that start in its chunk.  A run starts at monomer m
// when bond m-1 (cyclically) is non-zero and ends at the next non-zero bond.
__global__ void build_kernel(BuildArgs a)
{
    const int lane = threadIdx.x & 31;
    const int p = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (p >= a.P) return;                       // the whole warp leaves together
    const int L = a.L, N = a.N;
    const uint8_t* b = a.bonds + (size_t)p * N;
    const int t0 = a.start[3 * (size_t)p], u0 = a.start[3 * (size_t)p + 1], v0 = a.start[3 * (size_t)p + 2];
    const int C = (N + 31) / 32, m0 = lane * C, m1 = min(N, m0 + C);
    int bad = (t0 < 0 || u0 < 0 || v0 < 0 || t0 >= L || u0 >= L || v0 >= L) ? 1 : 0;
    if (a.linear && b[N - 1] != 15) bad = 1;
    int dt = 0, du = 0, dv = 0, nz = 0, firstnz = INT_MAX;
    for (int m = m0; m < m1; m++) {
        const uint32_t bm = b[m];
        if (bm > 15 || (bm && !elp_valid_bond(bm) && !(a.linear && m == N - 1))) bad = 1;
        dt += elp_bt(bm); du += elp_bu(bm); dv += elp_bv(bm);
        if (bm) {
            nz++;
            firstnz = min(firstnz, m);
        }
    }
    // inclusive prefix sums of the chunk displacements and of the non-zero count
    int it = dt, iu = du, iv = dv, inz = nz;
    for (int o = 1; o < 32; o <<= 1) {
        const int xt = __shfl_up_sync(0xffffffffu, it, o), xu = __shfl_up_sync(0xffffffffu, iu, o);
        const int xv = __shfl_up_sync(0xffffffffu, iv, o), xn = __shfl_up_sync(0xffffffffu, inz, o);
        if (lane >= o) { it += xt; iu += xu; iv += xv; inz += xn; }
    }
    const int tt = __shfl_sync(0xffffffffu, it, 31), tu = __shfl_sync(0xffffffffu, iu, 31);
    const int tv = __shfl_sync(0xffffffffu, iv, 31), tnz = __shfl_sync(0xffffffffu, inz, 31);
    // a ring closes and has two sites at least
    if (!a.linear && (wrap(t0 + tt, L) != t0 || wrap(u0 + tu, L) != u0 || wrap(v0 + tv, L) != v0 || tnz < 2)) bad = 1;
    if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) a.status[p] = 4;
        return;
    }
    // first non-zero bond in the lanes after this one, and in the whole chain
    int sm = firstnz;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_down_sync(0xffffffffu, sm, o);
        if (lane + o < 32) sm = min(sm, y);
    }
    int after = __shfl_down_sync(0xffffffffu, sm, 1);
    if (lane == 31) after = INT_MAX;
    const int first_all = __shfl_sync(0xffffffffu, sm, 0);
    // position of monomer m0 in the box; each bond then moves it by at most
    // one site per axis, wrapped without a division
    int t = wrap(t0 + it - dt, L), u = wrap(u0 + iu - du, L), v = wrap(v0 + iv - dv, L);
    int status = 0;
    for (int m = m0; m < m1; m++) {
        const uint32_t prev = b[m == 0 ? N - 1 : m - 1];
        if (prev) {   // a run starts at m
            int e = m;
            while (e < m1 && b[e] == 0) e++;
            if (e == m1) e = (after != INT_MAX) ? after : first_all + N;   // it ends in a later chunk, or wraps
            const int len = e - m + 1;
            const uint32_t bo = b[e % N];
            const uint32_t site = (uint32_t)t + (uint32_t)L * ((uint32_t)u + (uint32_t)L * (uint32_t)v);
            const int off0 = (N - m) % N;
            const bool head = off0 < len;   // this run holds monomer 0
            const uint32_t word = head ? (bo | ELP_LBIT | ((uint32_t)p << 5)) : (bo | ((uint32_t)len << ELP_CSHIFT));
            if (atomicCAS(&a.lat[site], 0u, word) != 0u) status = 3;
            if (head)
                *reinterpret_cast<uint4*>(a.rec + ELP_REC_WORDS * (size_t)p) =
                    make_uint4(site, (uint32_t)len, (uint32_t)off0, 0u);
        }
        const uint32_t bm = b[m];
        t += elp_bt(bm); u += elp_bu(bm); v += elp_bv(bm);
        t += t < 0 ? L : 0; t -= t >= L ? L : 0;
        u += u < 0 ? L : 0; u -= u >= L ? L : 0;
        v += v < 0 ? L : 0; v -= v >= L ? L : 0;
    }
    if (__any_sync(0xffffffffu, status)) {
        if (lane == 0) a.status[p] = 3;
    } else if (lane == 0) {
        a.status[p] = 0;
    }
}

// CreatePolymers (cpupol/efpol_init.c:239-283) written straight into site
// words: chain p's monomer 0 alone on its grid site (b_out +v, the label),
// monomers 1 .. N-1 stored on the next site along v (b_out -v closing a
// ring, or the end marker 0xf of a linear chain).
__global__ void init_kernel(uint32_t* lat, uint32_t* rec, int L, int N, int P, int linear, int delta, int nt, int nv)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int t = delta * (p % nt), u = delta * (p / nt / nv), v = (delta + 1) * ((p / nt) % nv);
    const uint32_t s0 = (uint32_t)t + (uint32_t)L * ((uint32_t)u + (uint32_t)L * (uint32_t)v);
    const uint32_t s1 = (uint32_t)t + (uint32_t)L * ((uint32_t)u + (uint32_t)L * (uint32_t)((v + 1) % L));
    lat[s0] = 0x4u | ELP_LBIT | ((uint32_t)p << 5);
    lat[s1] = (linear ? 0xfu : 0xbu) | ((uint32_t)(N - 1) << ELP_CSHIFT);
    *reinterpret_cast<uint4*>(rec + ELP_REC_WORDS * (size_t)p) = make_uint4(s0, 1u, 0u, 0u);
}

}  // namespace elp

elp_status elp_init_melt_device(uint32_t* lat, uint32_t* rec, int L, int N, int P, int linear, cudaStream_t s)
{
    int delta, nt, nv;
    if (elp_initial_grid(L, N, P, &delta, &nt, &nv))
        return elp_fail(ELP_ERR_ARG, "initial grid cannot hold %d rings of %d in L=%d", P, N, L);
    ELP_CUDA_TRY(cudaMemsetAsync(lat, 0, (size_t)L * L * L * sizeof(uint32_t), s));
    elp::init_kernel<<<(P + 127) / 128, 128, 0, s>>>(lat, rec, L, N, P, linear, delta, nt, nv);
    ELP_CUDA_TRY(cudaGetLastError());
    return ELP_OK;
}

elp_status elp_build_melt(uint32_t* lat, uint32_t* rec, int L, int N, int P, int linear, const int32_t* start,
                          const uint8_t* bonds, elp_walk_bufs* wb, cudaStream_t s)
{
    if (!lat || !rec || !start || !bonds || L < 1 || N < 1 || P < 1) return elp_fail(ELP_ERR_ARG, "bad argument");
    elp_status st = elp_walk_bufs_reserve(wb, P, N, 0);
    if (st) return st;
    const size_t S = (size_t)L * L * L;
    ELP_CUDA_TRY(cudaMemcpyAsync(wb->d_start, start, (size_t)P * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(wb->d_bonds, bonds, (size_t)P * N, cudaMemcpyHostToDevice, s));
    ELP_CUDA_TRY(cudaMemsetAsync(lat, 0, S * sizeof(uint32_t), s));
    elp::BuildArgs a;
    a.start = wb->d_start; a.bonds = wb->d_bonds; a.lat = lat; a.rec = rec; a.status = wb->d_status;
    a.L = L; a.N = N; a.P = P; a.linear = linear;
    elp::build_kernel<<<(unsigned)(((size_t)P * 32 + 127) / 128), 128, 0, s>>>(a);
    ELP_CUDA_TRY(cudaGetLastError());
    std::vector<int32_t> status((size_t)P);
    ELP_CUDA_TRY(cudaMemcpyAsync(status.data(), wb->d_status, (size_t)P * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    for (int p = 0; p < P; p++) {
        if (status[(size_t)p] == 3)
            return elp_fail(ELP_ERR_INTEGRITY, "chain %d: two rings or two runs of a ring share a site (code 3)", p);
        if (status[(size_t)p])
            return elp_fail(ELP_ERR_INTEGRITY, "chain %d: bad bond, ring not closed, or on a single site (code 4)", p);
    }
    return ELP_OK;
}
