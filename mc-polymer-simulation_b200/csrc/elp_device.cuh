// elp_device.cuh -- device core of the ELP sweep: counter RNG and the
// anchored single-monomer move.
//
// The move is the reference's efpol move (cpupol/efpol_lib.c:132-207): a
// monomer m with bonds (b_{m-1}, b_m) = (src1, src2) draws 4 random bits,
// looks up (dst1, dst2) in the transition table (cpupol/efpol_init.c:314-424)
// and moves to site(m-1) + dst1 when the target is free or part of its own
// chain.  What differs from efpol is only WHICH monomer is tried when: here a
// site P (the "anchor") tries the monomer whose predecessor sits on P --
// slot 0: the last monomer of P's run, slot 1: the first monomer of the next
// run.  A move and its reverse share the anchor and touch only P and sites
// one bond from P.
#pragma once
#include <stdint.h>

#include "elp_internal.h"

namespace elp {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint32_t bounded(uint32_t w, uint32_t n) { return __umulhi(w, n); }

__device__ __forceinline__ uint32_t word_of(uint4 v, int i)
{
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// One domain held in shared memory.
struct Dom {
    uint32_t* S;          // lattice words; index ox + x + sx*y + sxy*z
    const uint8_t* tab;   // 4096-entry table: dst1 | dst2<<4
    uint32_t* rec;        // chain records (global memory)
    int ox, sx, sxy;
    int x0, y0, z0, L;    // global coordinates of local (0,0,0); box edge
};

__device__ __forceinline__ uint32_t global_site(const Dom& D, int p)
{
    int q = p - D.ox;
    int z = q / D.sxy;
    int r = q - z * D.sxy;
    int y = r / D.sx;
    int x = r - y * D.sx;
    int L = D.L;
    int gx = D.x0 + x; gx -= (gx >= L) ? L : 0;
    int gy = D.y0 + y; gy -= (gy >= L) ? L : 0;
    int gz = D.z0 + z; gz -= (gz >= L) ? L : 0;
    return (uint32_t)gx + (uint32_t)L * ((uint32_t)gy + (uint32_t)L * (uint32_t)gz);
}

__device__ __forceinline__ uint32_t run_len(const Dom& D, uint32_t w)
{
    return (w & ELP_LBIT) ? D.rec[ELP_REC_WORDS * (w >> 5) + 1] : (w >> ELP_CSHIFT);
}

// General form of the move, including the bookkeeping of monomer 0's run.
// Taken only when a labelled run is involved (about one site per chain).
static __device__ __noinline__ int op_slow(const Dom& D, int p, const int* off, uint32_t s, uint32_t r4)
{
    uint32_t* S = D.S;
    uint32_t wP = S[p];
    uint32_t bo = wP & 15, cP = run_len(D, wP);
    uint32_t src1, src2, wB = 0, cB = 0;
    int pB = 0;
    if (s == 0) {
        if (cP < 2) return 0;
        src1 = 0;
        src2 = bo;
    } else {
        pB = p + off[bo];
        wB = S[pB];
        if (wB == ELP_WALL) return 0;
        cB = run_len(D, wB);
        src1 = bo;
        src2 = (cB >= 2) ? 0 : (wB & 15);
    }
    uint32_t e = D.tab[(src1 << 8) | (src2 << 4) | r4];
    uint32_t d1 = e & 15, d2 = e >> 4;
    if (!e) return 0;
    int pY = p + off[d1];
    uint32_t wY = S[pY];
    if (d1 && d2 && wY) return 0;
    if (!d2 && wY == ELP_WALL) return 0;
    uint32_t cN = d2 ? 0 : run_len(D, wY);

    uint32_t nPc = cP + (d1 == 0) - (src1 == 0);
    uint32_t wP2 = (d1 ? d1 : d2) | (nPc << ELP_CSHIFT);
    uint32_t wB2 = 0, wY2 = 0;
    if (s == 1 && src2 == 0) wB2 = (wB & 15) | ((cB - 1) << ELP_CSHIFT);
    if (d1 && d2) wY2 = d2 | ELP_CUNIT;
    else if (!d2) wY2 = (wY & 15) | ((cN + 1) << ELP_CSHIFT);

    int lab = -1;
    uint32_t chain = 0;
    if (wP & ELP_LBIT) { lab = 0; chain = wP >> 5; }
    else if (s == 1 && (wB & ELP_LBIT)) { lab = 1; chain = wB >> 5; }
    else if (!d2 && (wY & ELP_LBIT)) { lab = 2; chain = wY >> 5; }
    if (lab >= 0) {
        uint32_t* rc = D.rec + ELP_REC_WORDS * chain;
        uint32_t off0 = rc[2], noff;
        int nl;
        if (lab == 0) {
            nl = 0; noff = off0;
            if (s == 0 && off0 == cP - 1) { nl = 2; noff = 0; }
        } else if (lab == 1) {
            if (src2 == 0 && off0 > 0) { nl = 1; noff = off0 - 1; }
            else { nl = d1 ? 2 : 0; noff = d1 ? 0 : nPc - 1; }
        } else {
            nl = 2; noff = off0 + 1;
        }
        uint32_t* tgt = nl == 0 ? &wP2 : (nl == 1 ? &wB2 : &wY2);
        int ps = nl == 0 ? p : (nl == 1 ? pB : pY);
        rc[0] = global_site(D, ps);
        rc[1] = *tgt >> ELP_CSHIFT;
        rc[2] = noff;
        *tgt = (*tgt & 15) | ELP_LBIT | (chain << 5);
    }
    S[p] = wP2;
    if (s == 1) S[pB] = wB2;
    if (d1) S[pY] = wY2;
    return 1;
}

// The common case: no labelled run in the footprint.  Identical in effect to
// op_slow.  `off` holds the 16 shared-memory offsets of the bond codes for the
// anchor's boundary class.  rb: bit 0 slot, bits 1-4 table option.
__device__ __forceinline__ int op(const Dom& D, int p, const int* off, uint32_t rb)
{
    uint32_t* S = D.S;
    uint32_t wP = S[p];
    if (wP == 0) return 0;
    uint32_t s = rb & 1, r4 = (rb >> 1) & 15;
    uint32_t bo = wP & 15;
    uint32_t src1, src2, wB = 0;
    int pB = 0;
    uint32_t lab = wP & ELP_LBIT;
    if (s == 0) {
        if (!lab && wP < 2u * ELP_CUNIT) return 0;
        src1 = 0;
        src2 = bo;
    } else {
        pB = p + off[bo];
        wB = S[pB];
        if (wB == ELP_WALL) return 0;
        lab |= wB & ELP_LBIT;
        src1 = bo;
        src2 = (wB >= 2u * ELP_CUNIT) ? 0 : (wB & 15);
    }
    if (lab) return op_slow(D, p, off, s, r4);
    uint32_t e = D.tab[(src1 << 8) | (src2 << 4) | r4];
    if (!e) return 0;
    uint32_t d1 = e & 15, d2 = e >> 4;
    int pY = p + off[d1];
    uint32_t wY = S[pY];
    if (d2) {
        if (d1 && wY) return 0;          // new site must be free (walls are not)
    } else {
        if (wY == ELP_WALL) return 0;
        if (wY & ELP_LBIT) return op_slow(D, p, off, s, r4);
    }
    uint32_t cw = wP & ~15u;
    cw = (s == 0) ? cw - ELP_CUNIT : (d1 ? cw : cw + ELP_CUNIT);
    S[p] = cw | (d1 ? d1 : d2);
    if (s) S[pB] = (src2 == 0) ? wB - ELP_CUNIT : 0u;
    if (d1) S[pY] = d2 ? (d2 | ELP_CUNIT) : wY + ELP_CUNIT;
    return 1;
}

}  // namespace elp
