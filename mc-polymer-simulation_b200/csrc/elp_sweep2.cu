// elp_sweep2.cu -- specialised sweep kernels for the common domain shapes.
//
// Same schedule and results as the generic sweep_kernel (elp_sweep.cu); what
// changes is how the work is fed to the SM:
//   * tile edges and shared-memory strides are compile-time constants;
//   * the K anchors a thread owns in a substep are processed stage by stage
//     (all first loads, then all second loads, ...), so the dependent
//     shared-memory loads of independent moves overlap;
//   * monomer 0's runs are handled inline: while a tile is on chip each
//     labelled word carries its run length (bits 16-31) and a slot number
//     (bits 5-15) into a small shared-memory table {chain, offset | site};
//     the chain records in global memory are read when the tile is loaded and
//     written back when it is stored, so no move waits on global memory.  A
//     ring tile that holds more monomer-0 runs than the table (short rings
//     crowded together, as CreatePolymers leaves them) runs its substeps with
//     the general move of elp_device.cuh instead, which keeps that
//     bookkeeping in the chain records: slower, the same bits;
//   * a tile's rows are fetched in 16-byte cp.async granules.  The origin
//     shift makes a row start anywhere, so each row fetch takes the 16-byte
//     aligned span around the row (TX + 4 words) and the tile sits
//     sh = x0 mod 4 words into it; the words of the span outside the tile
//     become halo words.  Tiles go back with 16-byte stores (single words at
//     the ragged ends).  Rows are 16-byte aligned in shared memory, and the
//     threads of a warp take anchors from an 8 x 4 block of rows so that
//     their first loads hit 32 different banks;
//   * the grid is persistent over the tiles, and a launch of several steps
//     over a tiled box is cooperative, with a grid barrier between steps.
#include <cuda_runtime.h>
#include <math.h>

#include <atomic>

#include "elp_device.cuh"
#include "elp_kernels.h"

namespace elp {

__device__ __forceinline__ void cp_async4(uint32_t* sdst, const uint32_t* gsrc)
{
    uint32_t s = (uint32_t)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t* sdst, const uint32_t* gsrc)
{
    uint32_t s = (uint32_t)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Polls of the grid barrier before a wait gives up (about a second with the
// back-off below); a launch can ask for fewer (BatchLaunch.wait_polls).
constexpr uint32_t WAIT_POLLS = 1u << 24;

// Barrier over all CTAs of a cooperative launch: each CTA adds one to
// bar[0] and waits (bounded) until it reaches `target`.  The CTA's stores
// before it are visible to every CTA's loads after it (tiles are fetched
// with cp.async.cg and records with ld.global.cg, both through L2).
// Returns false, in every thread of the CTA, when the wait gave up.
// `arrive` false (a test) makes the CTA wait without adding its count.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t target, uint32_t polls, bool arrive)
{
    bool ok = true;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (arrive) atomicAdd(bar, 1u);
        for (uint32_t n = 0; ld_acquire_gpu(bar) < target; n++) {
            if (n >= polls) { ok = false; break; }
            __nanosleep(64);
        }
    }
    return __syncthreads_or(!ok) == 0;
}
// Last act of every CTA of a cooperative launch: the last one to leave
// zeroes the barrier counts for the next launch on the stream.
__device__ __forceinline__ void grid_exit(uint32_t* bar)
{
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(bar + 1, 1u) == gridDim.x - 1) {
        atomicExch(bar, 0u);
        atomicExch(bar + 1, 0u);
    }
}

template <int TX, int TY, int TZ, bool PER, int NC, int SX, int SXY, int CAP, int K, int MINB>
struct Shape {
    static constexpr int R = TY * TZ;
    static constexpr int A = R * (TX / NC);   // anchors per substep
    static constexpr int G = A / 4;           // Philox counters per substep group
    static constexpr int AT = A / K;          // threads that own anchors
    // Tiled domains: row y of plane z starts at OX + SX y + SXY z (16-byte
    // aligned) and holds the copied span of TX + 4 words, the tile at offset
    // sh in it; rows y = -1, TY and planes z = -1, TZ are halo, as is the
    // word before each row (the previous row's padding).
    static constexpr int SPAN = TX + 4;
    static constexpr int OX = PER ? 0 : SX + SXY + 4;
    static constexpr int WORDS = PER ? SXY * TZ : ((OX + SX * TY + SXY * TZ + SPAN + 3) & ~3);
    static constexpr int SITES = TX * TY * TZ;
    // threads of a warp take anchors from an 8 x 4 block of (y, z) rows
    static constexpr bool PERM = !PER && TY % 8 == 0 && TZ % 4 == 0 && AT % R == 0;
    // neighbour offsets: 27 boundary classes of a periodic box, one class in a tile
    static constexpr int NOFF = PER ? 27 * 16 : 16;
    // shared-memory word offsets: lattice, transition table (4096 bytes),
    // neighbour offsets (bytes, and for tiles in words too), colours, slot
    // tables, slot count, head-move rows, and the Philox words when threads
    // own < 4 anchors
    static constexpr int TABW = WORDS;
    static constexpr int OFFW = TABW + 1024;
    static constexpr int WOFFW = OFFW + NOFF;
    static constexpr int COLW = WOFFW + (PER ? 0 : 16);
    static constexpr int SHFW = COLW + 64;    // the step's domain shift (tiles), drawn by one warp
    static constexpr int SCHW = SHFW + 4;
    static constexpr int SSOW = SCHW + CAP;   // {offset of monomer 0 in its run (bits 0-15), site word (16-31)}
    static constexpr int NSLW = SSOW + CAP;
    static constexpr int HTABW = NSLW + 1;    // table rows (0xf, x): moves of a linear chain's monomer 0
    static constexpr int RNDW = (HTABW + 64 + 3) & ~3;
    static constexpr int NG = 2 * NC / 4;     // substep groups per step
    static constexpr size_t bytes_with(int groups) { return (size_t)(RNDW + (K < 4 ? groups * G * 4 : 0)) * 4; }
    // Philox words of threads that own < 4 anchors: in tiled domains, where
    // MINB CTAs still fit on an SM (228 KB, 1 KB reserved per CTA), all NG
    // groups of the step, drawn while the tile loads (PRE); else two buffers,
    // the next group's drawn during this one
    static constexpr bool PRE = !PER && K < 4 && (size_t)MINB * (bytes_with(NG) + 1024) <= 233472;
    static constexpr int TOTW = RNDW + (K < 4 ? (PRE ? NG : 2) * G * 4 : 0);
    static constexpr size_t BYTES = (size_t)TOTW * 4;
    static_assert(PER || (SX % 4 == 0 && SXY % 4 == 0 && SX >= SPAN + 1 && SXY >= SX * (TY + 2)),
                  "tiled rows: 16-byte aligned, room for the span and the halo word before it");
    static_assert(WORDS < 65536, "slot sites are 16-bit word indices");
    static_assert(BYTES <= 232448, "dynamic shared memory of one CTA");
};

constexpr uint32_t LMASK = 0xFFF0u;  // label bit + slot number
// Halo word of tiled domains: run length 1, b_out 3 (not a bond).  A slot-1
// move whose next run lies in the halo then looks up row (b_out(P), 3) of
// the table, which the kernel clears in its shared-memory copy, so the move
// is null without a separate test; a target in the halo is neither empty nor
// a run of the chain, so it is rejected as well.
constexpr uint32_t HWALL = ELP_CUNIT | 3u;

extern __shared__ __align__(16) uint32_t g_smem[];

// A labelled word (global form: chain id in bits 5-31) entering shared
// memory: claim a slot for the chain, keep {chain, offset | site} in the
// slot table and put the slot number and the run length into the word.  Past
// the table's capacity the word is left as it is (the tile then runs the
// general move).
template <int CAP>
__device__ __forceinline__ uint32_t take_slot(uint32_t wv, int idx, const uint32_t* rec, uint32_t* nslots,
                                              uint32_t* slot_chain, uint32_t* slot_so)
{
    const uint32_t slot = atomicAdd(nslots, 1u);
    if (slot >= (uint32_t)CAP) return wv;
    const uint32_t chain = wv >> 5;
    const uint4 rr = __ldcg(reinterpret_cast<const uint4*>(rec + ELP_REC_WORDS * (size_t)chain));
    slot_chain[slot] = chain;
    slot_so[slot] = rr.z | ((uint32_t)idx << 16);
    return (wv & 15) | ELP_LBIT | (slot << 5) | (rr.y << ELP_CSHIFT);
}

// Shared-memory word at byte offset b (offsets are kept in bytes so that a
// load or store needs no index scaling).
__device__ __forceinline__ uint32_t& SW(int b) { return *reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(g_smem) + b); }

// Monomer 0 sits in one of the runs a move touches (src: 0 the anchor's run,
// 1 the next run, 2 the target run): move its slot's site and offset along.
// Updates the new word (nP, nB or nY) that ends up holding monomer 0.
__device__ __forceinline__ void follow_label(uint32_t* slot_so, int p, int pB, int pY, uint32_t wP, uint32_t wB,
                                             uint32_t wY, uint32_t s, uint32_t d1, uint32_t& nP, uint32_t& nB,
                                             uint32_t& nY)
{
    const int src = (wP & ELP_LBIT) ? 0 : ((s && (wB & ELP_LBIT)) ? 1 : 2);
    const uint32_t lw = src == 0 ? wP : (src == 1 ? wB : wY);
    const uint32_t slot = (lw >> 5) & 0x7FFu;
    const uint32_t off0 = slot_so[slot] & 0xFFFFu;
    uint32_t noff;
    int nl;
    if (src == 0) {
        nl = 0; noff = off0;
        if (s == 0 && off0 == (wP >> ELP_CSHIFT) - 1) { nl = 2; noff = 0; }
    } else if (src == 1) {
        if (wB >= 2u * ELP_CUNIT && off0 > 0) { nl = 1; noff = off0 - 1; }
        else { nl = d1 ? 2 : 0; noff = d1 ? 0 : (nP >> ELP_CSHIFT) - 1; }
    } else {
        nl = 2; noff = off0 + 1;
    }
    const uint32_t lb = lw & LMASK;
    if (src == 0) nP &= ~LMASK; else if (src == 1) nB &= ~LMASK; else nY &= ~LMASK;
    if (nl == 0) nP |= lb; else if (nl == 1) nB |= lb; else nY |= lb;
    slot_so[slot] = noff | ((uint32_t)((nl == 0 ? p : (nl == 1 ? pB : pY)) >> 2) << 16);
}

// The Philox word of substep group k / 4 for this thread's anchors (counter
// word 3 gq).  Threads owning four anchors draw it themselves; with PRE all
// of the step's words were drawn while the tile loaded; otherwise G threads
// draw the next group's words into the other of two buffers while this group
// runs (read four barriers ago).
template <int K, bool PRE, int G, int NSUB>
__device__ __forceinline__ uint4 group_words(uint4* rnd, int k, uint32_t t, int d, int gq, uint2 key)
{
    if (K == 4) return philox(make_uint4(t, (uint32_t)d, (uint32_t)(k >> 2), (uint32_t)gq), key);
    if (PRE) return rnd[(k >> 2) * G + gq];
    const int cur = (k >> 2) & 1;
    const uint4 rw = rnd[cur * G + gq];
    if ((int)threadIdx.x < G && k + 4 < NSUB)
        rnd[(cur ^ 1) * G + threadIdx.x] = philox(make_uint4(t, (uint32_t)d, (uint32_t)(k >> 2) + 1u, threadIdx.x), key);
    return rw;
}

// All substeps of a ring tile whose monomer-0 runs outnumber the slots, with
// the general move (op: words in their global form, monomer 0's bookkeeping
// in the chain records, halo words ELP_WALL).  Not inlined: it runs rarely,
// and its registers stay out of the main substep loop.  Same anchors, random
// words and order as the main loop.  Returns this thread's accepted moves.
// This thread's anchors, passed by value so that the caller's copies stay in
// registers.
template <int K>
struct AnchorSet {
    int bse[K], rot[K], bsh[K];
};

template <int K, int NC, int WOFFW, bool PRE, int G>
__device__ __noinline__ uint32_t general_substeps(const Dom D, const AnchorSet<K> an, const uint32_t* col, uint4* rnd,
                                                  uint32_t t, int d, int gq, uint2 key)
{
    const int* bse = an.bse;
    const int* rot = an.rot;
    const int* bsh = an.bsh;
    const int* woffs = reinterpret_cast<const int*>(g_smem + WOFFW);
    uint32_t acc = 0;
    for (int k = 0; k < 2 * NC; k += 4) {
        const uint4 rw = group_words<K, PRE, G, 2 * NC>(rnd, k, t, d, gq, key);
        const uint32_t rws[4] = {rw.x, rw.y, rw.z, rw.w};
        for (int kk = 0; kk < 4; kk++) {
            const int c4 = (int)col[k + kk];
            for (int q = 0; q < K; q++) {
                int xr4 = c4 + rot[q];
                if ((NC & (NC - 1)) == 0) xr4 &= 4 * (NC - 1);
                else xr4 -= xr4 >= 4 * NC ? 4 * NC : 0;
                acc += (uint32_t)op(D, (bse[q] + xr4) >> 2, woffs, (rws[kk] >> bsh[q]) & 0xffu);
            }
            __syncthreads();
        }
    }
    return acc;
}

// The K anchors of one thread, one substep.  Returns accepted moves.  Anchor
// q takes its random byte at bit offset bsh[q] of the Philox word w: bit 0
// slot (0: the last monomer of P's run, 1: the first monomer of the next
// run), bits 1-4 table option.  Byte offsets: anchors base4 + 4 xr, colour
// c4 = 4 c, neighbour offsets at OFFW words; transition table (bytes) at
// TABW words.  `lin`: the melt holds linear chains (head moves of monomer 0).
template <int K, bool PER, int NC, int TABW, int OFFW, int HTABW>
__device__ __forceinline__ int substepK(uint32_t* slot_so, const int (&base4)[K], const int (&rot4)[K],
                                           const int (&clsyz)[K], const int (&xj4)[K], const int (&bsh)[K],
                                           const int (&an)[K], int c4, uint32_t w, int L, bool lin, uint32_t t, int d,
                                           int k, uint2 key)
{
    const uint8_t* tab = reinterpret_cast<const uint8_t*>(g_smem + TABW);
    const int* offs = reinterpret_cast<const int*>(g_smem + OFFW);
    int p[K], ob[K];
    uint32_t wP[K], rb[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
        int xr4 = c4 + rot4[q];
        if ((NC & (NC - 1)) == 0) xr4 &= 4 * (NC - 1);
        else xr4 -= xr4 >= 4 * NC ? 4 * NC : 0;
        p[q] = base4[q] + xr4;
        int cls = 0;
        if (PER) {
            int x4 = xr4 + xj4[q];
            cls = clsyz[q] + (x4 == 0 ? 0 : (x4 == 4 * (L - 1) ? 2 : 1));
        }
        ob[q] = 16 * cls;
        wP[q] = SW(p[q]);
        rb[q] = (w >> bsh[q]) & 0xffu;
    }
    int pB[K];
    uint32_t wB[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
        pB[q] = p[q] + offs[ob[q] + (wP[q] & 15)];
        wB[q] = SW(pB[q]);
    }
    uint32_t e[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
        const uint32_t s = rb[q] & 1, bo = wP[q] & 15;
        const bool c2 = (s ? wB[q] : wP[q]) >= 2u * ELP_CUNIT;
        const uint32_t src2 = s ? (c2 ? 0u : (wB[q] & 15)) : (c2 ? bo : 0u);
        e[q] = tab[((s ? bo : 0u) << 8) | (src2 << 4) | ((rb[q] >> 1) & 15)];
    }
    int pY[K];
    uint32_t wY[K];
#pragma unroll
    for (int q = 0; q < K; q++) {
        pY[q] = p[q] + offs[ob[q] + (e[q] & 15)];
        wY[q] = SW(pY[q]);
    }
    int acc = 0;
#pragma unroll
    for (int q = 0; q < K; q++) {
        const uint32_t d1 = e[q] & 15, d2 = e[q] >> 4, s = rb[q] & 1;
        const bool join = d2 == 0;  // m joins the front of the next run
        const bool ok = e[q] && (join ? wY[q] != HWALL : (d1 == 0 || wY[q] == 0));
        uint32_t nP = wP[q] & ~15u;
        nP = (s == 0) ? nP - ELP_CUNIT : (d1 ? nP : nP + ELP_CUNIT);
        nP |= d1 ? d1 : d2;
        uint32_t nB = (wB[q] >= 2u * ELP_CUNIT) ? wB[q] - ELP_CUNIT : 0u;
        uint32_t nY = d2 ? (d2 | ELP_CUNIT) : wY[q] + ELP_CUNIT;
        const uint32_t labs = (wP[q] | (s ? wB[q] : 0u) | (join ? wY[q] : 0u)) & ELP_LBIT;
        if (ok && labs) follow_label(slot_so, p[q], pB[q], pY[q], wP[q], wB[q], wY[q], s, d1, nP, nB, nY);
        if (ok && s) SW(pB[q]) = nB;
        if (ok && d1) SW(pY[q]) = nY;
        if (ok) SW(p[q]) = nP;
        wP[q] = ok ? nP : wP[q];
        acc += ok ? 1 : 0;
    }
    // linear chains: monomer 0 has no predecessor and moves about monomer 1,
    // tried at the anchor holding it after that anchor's regular attempt:
    // with probability 1/2 (bit 0 of its own Philox word) one option of row
    // (0xf, run length > 1 ? 0 : b_out) -- it leaves to the empty site P - u
    // (its bond to monomer 1 becoming u), or, alone on P, joins the next run
    if (lin) {
        const uint8_t* htab = reinterpret_cast<const uint8_t*>(g_smem + HTABW);
#pragma unroll
        for (int q = 0; q < K; q++) {
            const uint32_t w0 = wP[q];
            if (!(w0 & ELP_LBIT)) continue;
            const uint4 h = philox(make_uint4(t, (uint32_t)d, (uint32_t)k | ELP_STREAM_HEAD, (uint32_t)an[q]), key);
            if (!(h.x & 1)) continue;
            const uint32_t cP = w0 >> ELP_CSHIFT, bo = w0 & 15;
            const uint32_t e = htab[((cP >= 2 ? 0u : bo) << 4) | ((h.x >> 1) & 15)];
            if (!e) continue;
            const uint32_t d2 = e >> 4, slot = (w0 >> 5) & 0x7FFu;
            // monomer 0 of a linear chain is the first of its run: offset 0 stays
            if (cP >= 2) {
                const int pY = p[q] + offs[ob[q] + ((~d2) & 15u)];
                if (SW(pY) == 0) {
                    SW(pY) = d2 | (w0 & LMASK) | ELP_CUNIT;
                    SW(p[q]) = (w0 & ~LMASK) - ELP_CUNIT;
                    slot_so[slot] = (slot_so[slot] & 0xFFFFu) | ((uint32_t)(pY >> 2) << 16);
                    acc++;
                }
            } else {
                const int pB = p[q] + offs[ob[q] + bo];
                const uint32_t wB = SW(pB);
                if (wB != HWALL) {
                    SW(pB) = (wB + ELP_CUNIT) | (w0 & LMASK);
                    SW(p[q]) = 0;
                    slot_so[slot] = (slot_so[slot] & 0xFFFFu) | ((uint32_t)(pB >> 2) << 16);
                    acc++;
                }
            }
        }
    }
    return acc;
}

// K anchors per thread: K = 4 keeps four independent moves in flight per
// thread (instruction-level parallelism); K = 2 or 1 spreads a substep over
// more warps (latency hiding when a domain has few anchors per SM).  The
// random stream does not depend on K: anchor a = g + q * G always takes byte
// q of Philox word (k & 3) of counter {t, d, k / 4, g}.
template <int TX, int TY, int TZ, bool PER, int NC, int SX, int SXY, int CAP, int K, int THREADS, int MINB, bool LIN>
__global__ void __launch_bounds__(THREADS, MINB) sweep2_kernel(BatchLaunch a)
{
    using SH = Shape<TX, TY, TZ, PER, NC, SX, SXY, CAP, K, MINB>;
    static_assert(K == 1 || K == 2 || K == 4, "anchors per thread");
    static_assert(SH::A % 4 == 0 && SH::AT == THREADS && THREADS % 32 == 0, "every thread owns K anchors");
    static_assert(CAP <= 2048, "slot numbers are 11 bits");
    static_assert((2 * NC) % 4 == 0, "substeps come in groups of four");
    static_assert(THREADS % TX == 0, "tile columns are split evenly over the threads");
    constexpr int TABW = SH::TABW, OFFW = SH::OFFW, HTABW = SH::HTABW;
    uint32_t* S = g_smem;
    uint8_t* tab = reinterpret_cast<uint8_t*>(g_smem + TABW);
    int* offs = reinterpret_cast<int*>(g_smem + OFFW);
    uint32_t* col = g_smem + SH::COLW;
    uint32_t* shf = g_smem + SH::SHFW;
    uint32_t* slot_chain = g_smem + SH::SCHW;
    uint32_t* slot_so = g_smem + SH::SSOW;
    uint32_t* nslots = g_smem + SH::NSLW;
    uint4* rnd = reinterpret_cast<uint4*>(g_smem + SH::RNDW);
    const int tid = threadIdx.x;
    const int cx = tid % TX;  // the tile column this thread loads, scans and stores
    const int LP = TX;  // box edge of whole-box (periodic) domains

    // table words: entries 4i .. 4i+3 of row i / 4 = (src1 << 4) | src2.
    // Cleared: rows with a source that is no bond (3, 12: halo words) and
    // rows with src1 = 0xf (slot 1 at the last run of a linear chain, which
    // has no next run); rows (0xf, x) are kept apart for monomer-0 moves.
    for (int i = tid; i < 1024; i += THREADS) {
        const int s1 = i >> 6, s2 = (i >> 2) & 15;
        const bool nobond = s1 == 3 || s1 == 12 || s1 == 15 || s2 == 3 || s2 == 12;
        reinterpret_cast<uint32_t*>(tab)[i] = nobond ? 0u : a.table[i];
    }
    for (int i = tid; i < 64; i += THREADS) g_smem[HTABW + i] = a.table[960 + i];
    for (int i = tid; i < SH::NOFF; i += THREADS) {
        // whole box: class (cx, cy, cz) of the anchor on each axis (0 first
        // plane, 2 last, 1 inside) wraps the offsets; tiles: one class
        int cls = PER ? (i >> 4) : 13, b = i & 15;
        int dt = elp_bt(b), du = elp_bu(b), dv = elp_bv(b);
        if (PER) {
            int cx = cls % 3, cy = (cls / 3) % 3, cz = cls / 9;
            if (cx == 0 && dt < 0) dt = LP - 1;
            if (cx == 2 && dt > 0) dt = -(LP - 1);
            if (cy == 0 && du < 0) du = LP - 1;
            if (cy == 2 && du > 0) du = -(LP - 1);
            if (cz == 0 && dv < 0) dv = LP - 1;
            if (cz == 2 && dv > 0) dv = -(LP - 1);
        }
        offs[i] = 4 * (dt + SX * du + SXY * dv);   // bytes
        if (!PER) reinterpret_cast<int*>(g_smem + SH::WOFFW)[i] = dt + SX * du + SXY * dv;
    }
    if (!PER)
        for (int i = tid; i < SH::WORDS; i += THREADS) S[i] = HWALL;

    // Anchor an = g + q G of a substep takes byte q of Philox word g.  Thread
    // tid owns anchors an = tid + q AT, or with PERM the anchors of the same
    // x group whose row is the tid-th of the 8 x 4 row blocks.
    int base[K], rot[K], clsyz[K], xj[K], bsh[K], anq[K];
    int tperm = tid;
    if (SH::PERM) {
        const int r = tid % SH::R, lane = r & 31, w = r >> 5;
        const int y = (lane & 7) + 8 * (w % (TY / 8)), z = (lane >> 3) + 4 * (w / (TY / 8));
        tperm = tid - r + y + TY * z;
    }
    const int gq = tperm % SH::G;   // Philox counter word 3 of this thread's anchors
#pragma unroll
    for (int q = 0; q < K; q++) {
        int an = tperm + q * SH::AT;
        anq[q] = an;
        bsh[q] = 8 * (an / SH::G);
        int j = an / SH::R, row = an % SH::R;
        int y = row % TY, z = row / TY;
        int m = (2 * y + 3 * z) % NC;
        rot[q] = 4 * (m ? NC - m : 0);                       // bytes
        base[q] = 4 * (SH::OX + SX * y + SXY * z + NC * j);  // bytes
        int cy = y == 0 ? 0 : (y == LP - 1 ? 2 : 1);
        int cz = z == 0 ? 0 : (z == LP - 1 ? 2 : 1);
        clsyz[q] = PER ? (3 * cy + 9 * cz) : 13;
        xj[q] = 4 * NC * j;
    }
    const uint32_t step_dev = a.step_dev ? *a.step_dev : 0u;
    const uint32_t polls = a.wait_polls ? a.wait_polls : WAIT_POLLS;
    // Whole-box domains run their steps back to back on chip; tiled domains
    // move their tiles every step, so a launch of several steps takes its
    // steps one after another over all tiles, with a grid barrier between
    // steps (the launch is cooperative: all CTAs are resident).
    const int outer = PER ? 1 : a.nsteps, inner = PER ? a.nsteps : 1;

    for (int so = 0; so < outer; so++) {
    if (so > 0) {
        // a test may keep one CTA from arriving at the first barrier
        const bool arrive = !(so == 1 && (int)blockIdx.x + 1 == a.hold_cta1);
        if (!grid_barrier(a.grid_bar, gridDim.x * (uint32_t)so, polls, arrive)) {
            if (tid == 0) atomicOr(a.error, 4u);
            break;
        }
    }
    for (int it = blockIdx.x; it < a.nitems; it += gridDim.x) {
        const uint2 item = a.items[it];
        const BatchJob& J = a.jobs[item.x];
        const int d = (int)item.y;
        const int L = PER ? LP : J.L;
        uint32_t* lat = J.lat;
        uint32_t* rec = J.rec;
        const int nchains = J.nchains;
        const uint2 key = make_uint2(J.seed, J.salt);
        const bool lin = LIN && J.linear != 0;   // the ring instantiation has no monomer-0 moves
        const int ntx = J.ntx, nty = J.nty;
        Dom D;
        D.S = S; D.tab = tab; D.rec = rec;
        D.ox = SH::OX; D.sx = SX; D.sxy = SXY; D.L = L;
        D.x0 = 0; D.y0 = 0; D.z0 = 0;
        uint32_t accepted = 0;
        bool overflow = false, spill = false;
        int bse[K];   // anchor base byte offsets of this tile (plus its offset sh in the spans)
#pragma unroll
        for (int q = 0; q < K; q++) bse[q] = base[q];

        for (int st = 0; st < inner && !overflow; st++) {
            const uint32_t t = J.step0 + a.step_base + step_dev + (uint32_t)(so + st);
            if (!PER && tid < 32) {
                // one warp draws the step's domain shift for the whole CTA
                const uint4 sh = philox(make_uint4(t, 0, ELP_STREAM_SHIFT, 0), key);
                if (tid == 0) {
                    shf[0] = bounded(sh.x, TX);
                    shf[1] = bounded(sh.y, TY);
                    shf[2] = bounded(sh.z, TZ);
                }
            }
            if (st == 0) {
                __syncthreads();  // the previous item's stores have read shared memory; the shift is written
                if (!PER) {
                    D.x0 = (int)shf[0] + (d % ntx) * TX;
                    D.y0 = (int)shf[1] + ((d / ntx) % nty) * TY;
                    D.z0 = (int)shf[2] + (d / ntx / nty) * TZ;
                }
                if (tid == 0) *nslots = 0;
                const bool few = nchains <= THREADS;  // few rings: find monomer 0 through the records
                if (PER) {
                    // each thread owns one x column of the box: rows r = y + TY z
                    for (int r = tid / TX; r < SH::R; r += THREADS / TX) {
                        const int y = r % TY, z = r / TY;
                        cp_async4(S + cx + SX * y + SXY * z, lat + (uint32_t)(cx + L * (y + L * z)));
                    }
                    cp_async_wait_all();
                    __syncthreads();
                    if (!few) {
                        for (int r = tid / TX; r < SH::R; r += THREADS / TX) {
                            const int idx = cx + SX * (r % TY) + SXY * (r / TY);
                            const uint32_t wv = S[idx];
                            if (wv & ELP_LBIT) S[idx] = take_slot<CAP>(wv, idx, rec, nslots, slot_chain, slot_so);
                        }
                    }
                } else {
                    // rows r = y + TY z: the 16-byte aligned span [xa, xa + TX + 4)
                    // of the box row in 16-byte granules (a granule never
                    // straddles x = L: L and xa are multiples of 4)
                    const int xa = D.x0 & ~3, sh = D.x0 & 3;
                    D.ox = SH::OX + sh;
#pragma unroll
                    for (int q = 0; q < K; q++) bse[q] = base[q] + 4 * sh;
                    constexpr int CPR = SH::SPAN / 4;
                    for (int i = tid; i < SH::R * CPR; i += THREADS) {
                        const int r = i / CPR, c = i - r * CPR;
                        const int y = r % TY, z = r / TY;
                        int gy = D.y0 + y; gy -= gy >= L ? L : 0;
                        int gz = D.z0 + z; gz -= gz >= L ? L : 0;
                        int gx = xa + 4 * c; gx -= gx >= L ? L : 0;
                        cp_async16(S + SH::OX + SX * y + SXY * z + 4 * c, lat + (uint32_t)(gx + L * (gy + L * gz)));
                    }
                    // the step's Philox words while the rows are in flight
                    // (the same counters as the two-buffer schedule draws)
                    if (SH::PRE)
                        for (int i = tid; i < SH::NG * SH::G; i += THREADS)
                            rnd[i] = philox(make_uint4(t, (uint32_t)d, (uint32_t)(i / SH::G), (uint32_t)(i % SH::G)), key);
                    cp_async_wait_all();
                    __syncthreads();
                    // span words outside the tile become halo words; with many
                    // rings, monomer 0's runs are found in the same pass
                    for (int i = tid; i < SH::R * CPR; i += THREADS) {
                        const int r = i / CPR, c = i - r * CPR;
                        const int at = SH::OX + SX * (r % TY) + SXY * (r / TY) + 4 * c;
                        const int p0 = 4 * c - sh;  // tile column of the chunk's first word
                        uint4 v = *reinterpret_cast<const uint4*>(S + at);
                        const bool edge = p0 < 0 || p0 + 4 > TX;
                        if (edge) {
                            v.x = (unsigned)(p0 + 0) < (unsigned)TX ? v.x : HWALL;
                            v.y = (unsigned)(p0 + 1) < (unsigned)TX ? v.y : HWALL;
                            v.z = (unsigned)(p0 + 2) < (unsigned)TX ? v.z : HWALL;
                            v.w = (unsigned)(p0 + 3) < (unsigned)TX ? v.w : HWALL;
                        }
                        if (!few && ((v.x | v.y | v.z | v.w) & ELP_LBIT)) {
                            if (v.x & ELP_LBIT) v.x = take_slot<CAP>(v.x, at + 0, rec, nslots, slot_chain, slot_so);
                            if (v.y & ELP_LBIT) v.y = take_slot<CAP>(v.y, at + 1, rec, nslots, slot_chain, slot_so);
                            if (v.z & ELP_LBIT) v.z = take_slot<CAP>(v.z, at + 2, rec, nslots, slot_chain, slot_so);
                            if (v.w & ELP_LBIT) v.w = take_slot<CAP>(v.w, at + 3, rec, nslots, slot_chain, slot_so);
                            *reinterpret_cast<uint4*>(S + at) = v;
                        } else if (edge) {
                            *reinterpret_cast<uint4*>(S + at) = v;
                        }
                    }
                    if (few) __syncthreads();
                }
                if (few) {
                    for (int ch = tid; ch < nchains; ch += THREADS) {
                        const uint4 r = __ldcg(reinterpret_cast<const uint4*>(rec + ELP_REC_WORDS * (size_t)ch));
                        const int gx = (int)(r.x % (uint32_t)L), gy = (int)((r.x / (uint32_t)L) % (uint32_t)L),
                                  gz = (int)(r.x / ((uint32_t)L * L));
                        int x = gx - D.x0; x += x < 0 ? L : 0;
                        int y = gy - D.y0; y += y < 0 ? L : 0;
                        int z = gz - D.z0; z += z < 0 ? L : 0;
                        if (x < TX && y < TY && z < TZ) {
                            const uint32_t slot = atomicAdd(nslots, 1u);
                            if (slot < (uint32_t)CAP) {
                                const int idx = D.ox + x + SX * y + SXY * z;
                                slot_chain[slot] = (uint32_t)ch;
                                slot_so[slot] = r.z | ((uint32_t)idx << 16);
                                S[idx] = (S[idx] & 15) | ELP_LBIT | (slot << 5) | (r.y << ELP_CSHIFT);
                            }
                        }
                    }
                }
            }
            if (K < 4 && !SH::PRE && tid < SH::G) rnd[tid] = philox(make_uint4(t, (uint32_t)d, 0u, (uint32_t)tid), key);
            if (tid < (2 * NC + 3) / 4) {
                const uint4 cw = philox(make_uint4(t, (uint32_t)d, (uint32_t)tid | ELP_STREAM_COLOUR, 0), key);
                col[4 * tid + 0] = 4 * bounded(cw.x, NC);   // colours in bytes of x offset
                col[4 * tid + 1] = 4 * bounded(cw.y, NC);
                col[4 * tid + 2] = 4 * bounded(cw.z, NC);
                col[4 * tid + 3] = 4 * bounded(cw.w, NC);
            }
            __syncthreads();
            if (*nslots > (uint32_t)CAP) {
                if (PER || lin) {
                    // more monomer-0 runs than slots where the general move
                    // does not apply: leave this domain untouched, report
                    if (tid == 0) atomicOr(a.error, 1u);
                    overflow = true;
                    break;
                }
                // a crowded ring tile: words back to their global form (the
                // records still hold the runs' lengths and offsets), halo
                // words to the general move's wall
                spill = true;
                for (int sl = tid; sl < CAP; sl += THREADS) {
                    const int idx = (int)(slot_so[sl] >> 16);
                    S[idx] = (S[idx] & 15) | ELP_LBIT | (slot_chain[sl] << 5);
                }
                for (int i = tid; i < SH::WORDS; i += THREADS)
                    if (S[i] == HWALL) S[i] = ELP_WALL;
                __syncthreads();
            }
            if (!PER && spill) {
                AnchorSet<K> as;
#pragma unroll
                for (int q = 0; q < K; q++) {
                    as.bse[q] = bse[q];
                    as.rot[q] = rot[q];
                    as.bsh[q] = bsh[q];
                }
                accepted += general_substeps<K, NC, SH::WOFFW, SH::PRE, SH::G>(D, as, col, rnd, t, d, gq, key);
                continue;
            }
#pragma unroll 1
            for (int k = 0; k < 2 * NC; k += 4) {
                const uint4 rw = group_words<K, SH::PRE, SH::G, 2 * NC>(rnd, k, t, d, gq, key);
                const uint32_t rws[4] = {rw.x, rw.y, rw.z, rw.w};
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    accepted += (uint32_t)substepK<K, PER, NC, TABW, OFFW, HTABW>(
                        slot_so, bse, rot, clsyz, xj, bsh, anq, (int)col[k + kk], rws[kk], LP, lin, t, d, k + kk, key);
                    __syncthreads();
                }
            }
        }
        if (spill) {
            // the halo goes back to the form the slot-table path expects
            for (int i = tid; i < SH::WORDS; i += THREADS)
                if (S[i] == ELP_WALL) S[i] = HWALL;
        }
        if (!overflow) {
            const uint32_t ns = spill ? 0u : *nslots;   // a spilled tile's records are already written
            for (uint32_t sl = tid; sl < ns; sl += THREADS) {
                const uint32_t so16 = slot_so[sl];
                const int idx = (int)(so16 >> 16);
                const uint32_t wv = S[idx];
                const uint32_t chain = slot_chain[sl];
                *reinterpret_cast<uint4*>(rec + ELP_REC_WORDS * (size_t)chain) =
                    make_uint4(global_site(D, idx), wv >> ELP_CSHIFT, so16 & 0xFFFFu, 0u);
                S[idx] = (wv & 15) | ELP_LBIT | (chain << 5);
            }
            __syncthreads();
            if (PER) {
                for (int r = tid / TX; r < SH::R; r += THREADS / TX) {
                    const int y = r % TY, z = r / TY;
                    lat[(uint32_t)(cx + L * (y + L * z))] = S[cx + SX * y + SXY * z];
                }
            } else {
                // 16-byte stores of the span's chunks inside the tile, single
                // words at its ragged ends (a chunk never straddles x = L)
                const int xa = D.x0 & ~3, sh = D.x0 & 3;
                constexpr int CPR = SH::SPAN / 4;
                for (int i = tid; i < SH::R * CPR; i += THREADS) {
                    const int r = i / CPR, c = i - r * CPR;
                    const int y = r % TY, z = r / TY;
                    int gy = D.y0 + y; gy -= gy >= L ? L : 0;
                    int gz = D.z0 + z; gz -= gz >= L ? L : 0;
                    int gx = xa + 4 * c; gx -= gx >= L ? L : 0;
                    uint32_t* g = lat + (uint32_t)(gx + L * (gy + L * gz));
                    const uint32_t* cp = S + SH::OX + SX * y + SXY * z + 4 * c;
                    const int p0 = 4 * c - sh;
                    if (p0 >= 0 && p0 + 4 <= TX) {
                        *reinterpret_cast<uint4*>(g) = *reinterpret_cast<const uint4*>(cp);
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            if ((unsigned)(p0 + k) < (unsigned)TX) g[k] = cp[k];
                    }
                }
            }
        }
        if (J.acc) {
            unsigned long long v = (unsigned long long)accepted;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0 && v) atomicAdd(J.acc, v);
        }
    }
    }
    if (!PER && a.nsteps > 1) grid_exit(a.grid_bar);
}

}  // namespace elp

// ---- dispatch ----------------------------------------------------------------
namespace {
// Resident CTAs per SM of one kernel, per device (a cooperative launch is
// sized by it); 0 until the group set-up on that device has asked.
constexpr int MAX_DEVICES = 64;
}

template <int TX, int TY, int TZ, bool PER, int NC, int SX, int SXY, int CAP, int K, int THREADS, int MINB, bool LIN>
static cudaError_t launch2(const Sweep2Launch* l, cudaStream_t s)
{
    using SH = elp::Shape<TX, TY, TZ, PER, NC, SX, SXY, CAP, K, MINB>;
    auto k = elp::sweep2_kernel<TX, TY, TZ, PER, NC, SX, SXY, CAP, K, THREADS, MINB, LIN>;
    static std::atomic<int> per_sm[MAX_DEVICES];   // zero-initialised (static storage)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    if (l->check_only) {
        // expected monomer-0 runs per domain must stay far inside the slot table
        const double m = l->max_runs_per_domain;
        if (!(PER ? m <= CAP : m + 8.0 * sqrt(m) + 16.0 <= CAP)) return cudaErrorNotSupported;
        // set the shared-memory limit and size the grid here, outside any
        // stream capture, once per device (groups are committed often in the
        // serving loop)
        if (per_sm[dev].load() < 1) {
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::BYTES);
            int n = 0;
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, THREADS, SH::BYTES);
            if (e != cudaSuccess) return e;
            if (n < 1) return cudaErrorNotSupported;
            per_sm[dev].store(n);
        }
        const_cast<Sweep2Launch*>(l)->threads_out = THREADS;
        const_cast<Sweep2Launch*>(l)->smem_out = SH::BYTES;
        return cudaSuccess;
    }
    int grid = l->args.nitems;
    if (PER || l->args.nsteps <= 1) {
        if (grid > l->nsm * MINB) grid = l->nsm * MINB;
        if (grid < 1) return cudaSuccess;
        k<<<grid, THREADS, SH::BYTES, s>>>(l->args);
        return cudaGetLastError();
    }
    // tiled, several steps: a cooperative launch (every CTA resident, or an
    // error) of at most as many CTAs as fit on the device at once
    const int per = per_sm[dev].load();
    if (per < 1) return cudaErrorNotSupported;
    if (grid > l->nsm * per) grid = l->nsm * per;
    if (grid < 1) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SH::BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, l->args);
}

// Launch (or, with check_only, test) the specialised kernel for a shape.
// Returns cudaErrorNotSupported when none fits (the caller then uses the
// generic kernel).
extern "C" cudaError_t elp_launch_sweep2(const Sweep2Launch* l, cudaStream_t s)
{
    const elp_geometry& g = l->geom;
    if (l->args.nsteps > 1 && !g.periodic && !l->args.grid_bar) return cudaErrorNotSupported;
// shape: tile edges, whole box or tiled, colour modulus, shared-memory
// strides, slot capacity, anchors per thread, threads, min blocks per SM
#define SHAPE(X_, Y_, Z_, PER_, NC_, SX_, SXY_, CAP_, K_, THR_, MINB_)                                        \
    if (g.tx == X_ && g.ty == Y_ && g.tz == Z_ && g.periodic == PER_ && g.ncol == NC_ && l->sx == SX_ &&       \
        l->sxy == SXY_)                                                                                        \
        return l->linear ? launch2<X_, Y_, Z_, PER_, NC_, SX_, SXY_, CAP_, K_, THR_, MINB_, true>(l, s)        \
                         : launch2<X_, Y_, Z_, PER_, NC_, SX_, SXY_, CAP_, K_, THR_, MINB_, false>(l, s);
    SHAPE(32, 32, 32, 0, 16, 40, 1364, 1792, 2, 1024, 1)
    SHAPE(32, 32, 16, 0, 16, 40, 1364, 1024, 1, 1024, 1)
    SHAPE(32, 16, 16, 0, 16, 40, 724, 1024, 1, 512, 2)
    SHAPE(16, 16, 16, 0, 16, 24, 444, 512, 1, 256, 4)
    SHAPE(48, 24, 24, 0, 16, 56, 1456, 2048, 2, 864, 1)
    SHAPE(16, 16, 16, 1, 16, 16, 256, 2048, 1, 256, 1)
    SHAPE(32, 32, 32, 1, 16, 33, 1056, 2048, 2, 1024, 1)
    SHAPE(24, 24, 24, 1, 24, 24, 576, 2048, 1, 576, 1)
#undef SHAPE
    return cudaErrorNotSupported;
}
