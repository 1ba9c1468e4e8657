// elp_sweep.cu -- the sm_100a sweep kernel.
//
// Replaces the reference's polmove launch loop (gpupol2/gpupol_cuda.cu:114-152,
// gpupol2/ringpol3.cu:221-327) with a kernel that runs the reference CPU
// engine's move set (cpupol/efpol_lib.c:132-207) under a conflict-free,
// replayable schedule:
//
//   * one CTA per domain; the domain's site words live in shared memory;
//   * tiled boxes: the domain is a tile of the box plus a one-site halo of
//     wall words (moves that would touch another tile are rejected), and the
//     tile grid is shifted by a random vector every step (one step per
//     launch); periodic boxes: the whole box is one domain with wrap-around
//     neighbour offsets and stays on chip for any number of steps;
//   * a step is 2n substeps; substep k activates the sites whose colour
//     (x + 2y + 3z) mod n equals a random c_k -- their radius-1 footprints
//     never overlap (n = 16: 13 would be a perfect code) -- and every active
//     site makes one anchored move attempt (elp_device.cuh);
//   * randomness is Philox4x32-10 keyed by (seed, salt) with counters built
//     from (step, domain, substep, anchor group), so a host replay
//     reproduces every word bit for bit.
#include <cuda_runtime.h>

#include "elp_device.cuh"
#include "elp_kernels.h"

namespace elp {

struct RowInfo {
    int base;      // x + base = anchor index for x (smem, incl. ox)
    int rot;       // (-(2y + 3z)) mod n
    int clsyz;     // boundary class part from y, z (periodic)
    int j;         // which n-block of the row
};

__global__ void __launch_bounds__(1024) sweep_kernel(SweepArgs a)
{
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* S = smem;
    uint8_t* tab = reinterpret_cast<uint8_t*>(smem + a.words);
    int* offs = reinterpret_cast<int*>(tab + 4096);
    uint32_t* col = reinterpret_cast<uint32_t*>(offs + 27 * 16);

    const int tid = threadIdx.x, nthr = blockDim.x;
    const int d = blockIdx.x;
    const int n = a.ncol;
    const int tx = a.tx, ty = a.ty, tz = a.tz, L = a.L;
    const int R = ty * tz;
    const int G = a.groups;
    const uint2 key = make_uint2(a.seed, a.salt);

    // transition table and neighbour offsets
    for (int i = tid; i < 1024; i += nthr) reinterpret_cast<uint32_t*>(tab)[i] = a.table[i];
    for (int i = tid; i < 27 * 16; i += nthr) {
        int cls = i >> 4, b = i & 15;
        int dt = elp_bt(b), du = elp_bu(b), dv = elp_bv(b);
        if (a.periodic) {
            int cx = cls % 3, cy = (cls / 3) % 3, cz = cls / 9;
            if (cx == 0 && dt < 0) dt = L - 1;
            if (cx == 2 && dt > 0) dt = -(L - 1);
            if (cy == 0 && du < 0) du = L - 1;
            if (cy == 2 && du > 0) du = -(L - 1);
            if (cz == 0 && dv < 0) dv = L - 1;
            if (cz == 2 && dv > 0) dv = -(L - 1);
        }
        offs[i] = dt + a.sx * du + a.sxy * dv;
    }

    // this thread's anchor group g = tid: anchors a = g + q*G, q = 0..3
    RowInfo ri[4];
    const bool active = tid < G;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int an = tid + q * G;
        int j = an / R, row = an - (an / R) * R;
        int y = row % ty, z = row / ty;
        int m = (2 * y + 3 * z) % n;
        ri[q].rot = m ? n - m : 0;
        ri[q].base = a.ox + a.sx * y + a.sxy * z + n * j;
        int cy = y == 0 ? 0 : (y == L - 1 ? 2 : 1);
        int cz = z == 0 ? 0 : (z == L - 1 ? 2 : 1);
        ri[q].clsyz = a.periodic ? (3 * cy + 9 * cz) : 13;
        ri[q].j = j;
    }

    Dom D;
    D.S = S; D.tab = tab; D.rec = a.rec;
    D.ox = a.ox; D.sx = a.sx; D.sxy = a.sxy; D.L = L;
    D.x0 = 0; D.y0 = 0; D.z0 = 0;

    const int ntx = L / tx, nty = L / ty;
    const int warp = tid >> 5, lane = tid & 31, nwarp = nthr >> 5;
    uint32_t accepted = 0;

    for (int st = 0; st < a.nsteps; st++) {
        const uint32_t t = (uint32_t)(a.step0 + st);
        if (!a.periodic) {
            uint4 sh = philox(make_uint4(t, 0, ELP_STREAM_SHIFT, 0), key);
            D.x0 = (int)bounded(sh.x, tx) + (d % ntx) * tx;
            D.y0 = (int)bounded(sh.y, ty) + ((d / ntx) % nty) * ty;
            D.z0 = (int)bounded(sh.z, tz) + (d / ntx / nty) * tz;
        }
        if (st == 0 || !a.periodic) {
            if (!a.periodic)
                for (int i = tid; i < a.words; i += nthr) S[i] = ELP_WALL;
            __syncthreads();
            for (int r = warp; r < R; r += nwarp) {
                int y = r % ty, z = r / ty;
                int gy = D.y0 + y; gy -= gy >= L ? L : 0;
                int gz = D.z0 + z; gz -= gz >= L ? L : 0;
                const uint32_t* src = a.lat + (size_t)L * ((size_t)gy + (size_t)L * gz);
                uint32_t* dst = S + a.ox + a.sx * y + a.sxy * z;
                for (int x = lane; x < tx; x += 32) {
                    int gx = D.x0 + x; gx -= gx >= L ? L : 0;
                    dst[x] = src[gx];
                }
            }
        }
        if (tid < (2 * n + 3) / 4) {
            uint4 cw = philox(make_uint4(t, (uint32_t)d, (uint32_t)tid | ELP_STREAM_COLOUR, 0), key);
            col[4 * tid + 0] = bounded(cw.x, n);
            col[4 * tid + 1] = bounded(cw.y, n);
            col[4 * tid + 2] = bounded(cw.z, n);
            col[4 * tid + 3] = bounded(cw.w, n);
        }
        __syncthreads();

        uint4 rw = make_uint4(0, 0, 0, 0);
        for (int k = 0; k < 2 * n; k++) {
            if (active) {
                if ((k & 3) == 0) rw = philox(make_uint4(t, (uint32_t)d, (uint32_t)(k >> 2), (uint32_t)tid), key);
                const uint32_t w = word_of(rw, k & 3);
                const int c = (int)col[k];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    int xr = c + ri[q].rot;
                    xr -= xr >= n ? n : 0;
                    int x = xr + n * ri[q].j;
                    int cls = ri[q].clsyz;
                    if (a.periodic) cls += x == 0 ? 0 : (x == L - 1 ? 2 : 1);
                    accepted += op(D, ri[q].base + xr, offs + 16 * cls, (w >> (8 * q)) & 0xffu);
                    (void)x;
                }
            }
            __syncthreads();
        }

        if (st == a.nsteps - 1 || !a.periodic) {
            for (int r = warp; r < R; r += nwarp) {
                int y = r % ty, z = r / ty;
                int gy = D.y0 + y; gy -= gy >= L ? L : 0;
                int gz = D.z0 + z; gz -= gz >= L ? L : 0;
                uint32_t* dstg = a.lat + (size_t)L * ((size_t)gy + (size_t)L * gz);
                const uint32_t* src = S + a.ox + a.sx * y + a.sxy * z;
                for (int x = lane; x < tx; x += 32) {
                    int gx = D.x0 + x; gx -= gx >= L ? L : 0;
                    dstg[gx] = src[x];
                }
            }
            if (!a.periodic) __syncthreads();
        }
    }
    if (a.accepted) {
        for (int o = 16; o > 0; o >>= 1) accepted += __shfl_xor_sync(0xffffffffu, accepted, o);
        if (lane == 0 && accepted) atomicAdd(a.accepted, (unsigned long long)accepted);
    }
}

}  // namespace elp

extern "C" cudaError_t elp_launch_sweep(const SweepArgs* a, int ndomains, int threads, size_t smem, cudaStream_t s)
{
    static int attr_set = 0;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(elp::sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        attr_set = 1;
    }
    elp::sweep_kernel<<<ndomains, threads, smem, s>>>(*a);
    return cudaGetLastError();
}
