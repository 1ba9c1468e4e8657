// elp_build.cu -- site words and chain records built on the device from
// chains (start site of monomer 0 plus N bond codes per chain, the content
// of a TUV file, cpupol/efpol_io.c:3-47).
//
// The load path ships only the chains to the device (12 P + N P bytes) and
// builds the lattice there, instead of building L^3 site words on the host
// and copying them.  One thread per chain checks its bonds (valid codes; a
// ring closes, a linear chain ends in the marker 0xf), walks its runs from
// the first monomer whose predecessor bond is non-zero and claims each run's
// site with a compare-and-swap on the zeroed lattice: a site claimed twice
// means two runs on one site, efpol's CheckIntegrity code 3
// (cpupol/efpol_io.c:182-187); a bad bond or an open ring is code 4.
#include <cuda_runtime.h>

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

__global__ void build_kernel(BuildArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.P) return;
    const int L = a.L, N = a.N;
    const uint8_t* b = a.bonds + (size_t)p * N;
    const int t0 = a.start[3 * (size_t)p], u0 = a.start[3 * (size_t)p + 1], v0 = a.start[3 * (size_t)p + 2];
    int status = 0;
    if (t0 < 0 || u0 < 0 || v0 < 0 || t0 >= L || u0 >= L || v0 >= L) status = 4;
    if (!status && a.linear && b[N - 1] != 15) status = 4;
    int nz = 0, t = t0, u = u0, v = v0;
    for (int m = 0; m < N && !status; m++) {
        const uint32_t bm = b[m];
        if (bm > 15 || (bm && !elp_valid_bond(bm) && !(a.linear && m == N - 1))) status = 4;
        t += elp_bt(bm); u += elp_bu(bm); v += elp_bv(bm);
        nz += bm ? 1 : 0;
    }
    if (!status && !a.linear && (wrap(t, L) != t0 || wrap(u, L) != u0 || wrap(v, L) != v0 || nz < 2)) status = 4;
    if (!status) {
        // runs start at monomers whose predecessor's bond is non-zero
        int first = 0;
        while (!b[(first + N - 1) % N]) first++;
        t = t0; u = u0; v = v0;
        for (int m = 0; m < first; m++) { t += elp_bt(b[m]); u += elp_bu(b[m]); v += elp_bv(b[m]); }
        int m = first, done = 0;
        while (done < N) {
            int len = 1;
            while (len < N && b[(m + len - 1) % N] == 0) len++;
            const uint32_t site =
                (uint32_t)wrap(t, L) + (uint32_t)L * ((uint32_t)wrap(u, L) + (uint32_t)L * (uint32_t)wrap(v, L));
            const uint32_t bo = b[(m + len - 1) % N];
            const int off0 = (N - m) % N;
            const bool head = off0 < len;   // this run holds monomer 0
            const uint32_t word = head ? (bo | ELP_LBIT | ((uint32_t)p << 5)) : (bo | ((uint32_t)len << ELP_CSHIFT));
            if (atomicCAS(&a.lat[site], 0u, word) != 0u) {
                status = 3;
                break;
            }
            if (head)
                *reinterpret_cast<uint4*>(a.rec + ELP_REC_WORDS * (size_t)p) =
                    make_uint4(site, (uint32_t)len, (uint32_t)off0, 0u);
            t += elp_bt(bo); u += elp_bu(bo); v += elp_bv(bo);
            done += len;
            m = (m + len) % N;
        }
    }
    a.status[p] = status;
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
    elp::build_kernel<<<(P + 127) / 128, 128, 0, s>>>(a);
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
