// elp_observe.cu -- in-situ observables of a melt, computed on the device.
//
// One thread per ring walks the ring from monomer 0's run (walk_kernel
// follows the same runs, one warp per ring) and accumulates exact integer sums over its monomers, positions
// taken relative to monomer 0's site and unwrapped along the ring:
//   St, Su, Sv    sums of the lattice coordinates (t, u, v)
//   Sq            sum of x^2 + y^2 + z^2 with x = t+u-v, y = t-u, z = v
//   runs          occupied sites of the ring (zero bonds = N - runs; a
//                 linear chain ends in the run whose b_out is the marker 0xf)
// and a block-level histogram of run lengths (monomers per occupied site).
// Only these P x 48 bytes go to the host, where the centre of mass, the
// radius of gyration and the stored-length fraction are formed exactly as
// ComputeCMS / ComputeGyration / ComputeSL (analysis/mode_compute.c:145-217)
// form them from the PTL positions of LoadPTL (analysis/mode_io.c:509-606).
#include <cuda_runtime.h>
#include <string.h>

#include <vector>

#include "elp_common.h"
#include "elp_internal.h"
#include "elp_kernels.h"

namespace elp {

struct ObsArgs {
    const uint32_t* lat;
    const uint32_t* rec;
    int L, N, P, nbins, linear;
    unsigned long long* out;    // [P][6]: St, Su, Sv, Sq, runs | status << 32, site of monomer 0
    unsigned long long* hist;   // [nbins]
};

__global__ void observe_kernel(ObsArgs a)
{
    __shared__ unsigned long long hist[ELP_OBS_MAX_BINS];
    for (int i = threadIdx.x; i < a.nbins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < a.P) {
        const int L = a.L, N = a.N;
        const size_t S = (size_t)L * L * L;
        const uint32_t site = a.rec[ELP_REC_WORDS * p], cnt = a.rec[ELP_REC_WORDS * p + 1],
                       off = a.rec[ELP_REC_WORDS * p + 2];
        int bad = (site >= S || off >= cnt || cnt == 0 || (a.linear && off != 0)) ? 1 : 0;
        if (!bad) {
            const uint32_t w = a.lat[site];
            if (!(w & ELP_LBIT) || (w >> 5) != (uint32_t)p) bad = 1;
        }
        long long st = 0, su = 0, sv = 0;
        unsigned long long sq = 0, runs = 0;
        int dt = 0, du = 0, dv = 0;    // position of the current run relative to monomer 0's site
        long mono = 0;
        uint32_t here = cnt - off, cur = site, len = cnt;
        // the current run's site in box coordinates, stepped without a division
        int t = (int)(site % (uint32_t)L), u = (int)((site / (uint32_t)L) % (uint32_t)L),
            v = (int)(site / ((uint32_t)L * L));
        while (!bad) {
            const uint32_t bo = a.lat[cur] & 15;
            const bool end = a.linear && bo == 15;   // last run of a linear chain
            if (!(elp_valid_bond(bo) || end) || mono + (long)here > (long)N) { bad = 1; break; }
            const long long x = dt + du - dv, y = dt - du, z = dv;
            st += (long long)here * dt;
            su += (long long)here * du;
            sv += (long long)here * dv;
            sq += (unsigned long long)here * (unsigned long long)(x * x + y * y + z * z);
            mono += here;
            runs++;
            atomicAdd(&hist[(len < (uint32_t)a.nbins ? len : (uint32_t)a.nbins) - 1], 1ull);
            if (end) break;
            // next run
            t += elp_bt(bo); u += elp_bu(bo); v += elp_bv(bo);
            dt += elp_bt(bo); du += elp_bu(bo); dv += elp_bv(bo);
            t += t < 0 ? L : 0; t -= t >= L ? L : 0;
            u += u < 0 ? L : 0; u -= u >= L ? L : 0;
            v += v < 0 ? L : 0; v -= v >= L ? L : 0;
            cur = (uint32_t)t + (uint32_t)L * ((uint32_t)u + (uint32_t)L * (uint32_t)v);
            const uint32_t wn = a.lat[cur];
            if (!wn) { bad = 1; break; }
            if (cur == site) break;
            if (wn & ELP_LBIT) { bad = 1; break; }
            here = len = wn >> ELP_CSHIFT;
            if (here == 0 || runs >= (unsigned long long)N) { bad = 1; break; }
        }
        if (!bad) {
            // monomers N-off .. N-1: the rest of monomer 0's run, reached again after the whole ring
            const long long x = dt + du - dv, y = dt - du, z = dv;
            st += (long long)off * dt;
            su += (long long)off * du;
            sv += (long long)off * dv;
            sq += (unsigned long long)off * (unsigned long long)(x * x + y * y + z * z);
            mono += off;
            if (mono != N) bad = 1;
        }
        unsigned long long* o = a.out + 6 * (size_t)p;
        o[0] = (unsigned long long)st;
        o[1] = (unsigned long long)su;
        o[2] = (unsigned long long)sv;
        o[3] = sq;
        o[4] = runs | ((unsigned long long)(bad ? 4 : 0) << 32);
        o[5] = site;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.nbins; i += blockDim.x)
        if (hist[i]) atomicAdd(&a.hist[i], hist[i]);
}

}  // namespace elp

elp_status elp_observe_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                            double* cms_tuv, double* rg2, double* sl, uint64_t* run_hist, int nbins, cudaStream_t s)
{
    if (nbins < 0 || nbins > ELP_OBS_MAX_BINS)
        return elp_fail(ELP_ERR_ARG, "nbins must be in [0, %d]", ELP_OBS_MAX_BINS);
    if (run_hist && nbins < 1) return elp_fail(ELP_ERR_ARG, "run_hist needs nbins >= 1");
    const size_t need = (size_t)P * 6 + ELP_OBS_MAX_BINS;
    if (need > b->cap_obs) {
        cudaFree(b->d_obs);
        b->d_obs = nullptr;
        ELP_CUDA_TRY(cudaMalloc((void**)&b->d_obs, need * sizeof(unsigned long long)));
        b->bytes += (need - b->cap_obs) * sizeof(unsigned long long);
        b->cap_obs = need;
    }
    elp::ObsArgs a;
    a.lat = lat; a.rec = rec; a.L = L; a.N = N; a.P = P; a.linear = linear;
    a.nbins = nbins > 0 ? nbins : 1;
    a.out = b->d_obs;
    a.hist = b->d_obs + (size_t)P * 6;
    ELP_CUDA_TRY(cudaMemsetAsync(a.hist, 0, ELP_OBS_MAX_BINS * sizeof(unsigned long long), s));
    elp::observe_kernel<<<(P + 127) / 128, 128, 0, s>>>(a);
    ELP_CUDA_TRY(cudaGetLastError());
    std::vector<unsigned long long> o((size_t)P * 6);
    std::vector<unsigned long long> h(ELP_OBS_MAX_BINS);
    ELP_CUDA_TRY(cudaMemcpyAsync(o.data(), a.out, o.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(h.data(), a.hist, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    for (int p = 0; p < P; p++)
        if (o[6 * (size_t)p + 4] >> 32)
            return elp_fail(ELP_ERR_INTEGRITY, "ring %d cannot be walked", p);
    const double n = (double)N;
    for (int p = 0; p < P; p++) {
        const unsigned long long* r = &o[6 * (size_t)p];
        const long long st = (long long)r[0], su = (long long)r[1], sv = (long long)r[2];
        const uint32_t site = (uint32_t)r[5];
        if (cms_tuv) {
            cms_tuv[3 * (size_t)p + 0] = (double)(site % (uint32_t)L) + (double)st / n;
            cms_tuv[3 * (size_t)p + 1] = (double)((site / (uint32_t)L) % (uint32_t)L) + (double)su / n;
            cms_tuv[3 * (size_t)p + 2] = (double)(site / ((uint32_t)L * L)) + (double)sv / n;
        }
        if (rg2) {
            // Rg^2 = (N Sq - |S_xyz|^2) / (2 N^2), the numerator exact in 128 bits
            const __int128 sx = (__int128)st + su - sv, sy = (__int128)st - su, sz = sv;
            const __int128 num = (__int128)N * (__int128)r[3] - (sx * sx + sy * sy + sz * sz);
            rg2[p] = (double)num / (2.0 * n * n);
        }
        // zero bonds over the chain's bonds (a linear chain's end marker is none)
        if (sl) sl[p] = (double)((unsigned long long)N - (r[4] & 0xffffffffull)) / (linear ? n - 1.0 : n);
    }
    if (run_hist)
        for (int i = 0; i < nbins; i++) run_hist[i] = h[(size_t)i];
    return ELP_OK;
}
