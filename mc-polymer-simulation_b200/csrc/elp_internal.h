// elp_internal.h -- shared definitions of the ELP sweep engine (host + device).
//
// Site word (uint32, one per lattice site, index t + L*(u + L*v)):
//   bits 0-3   b_out: FCC bond code from the last monomer of the run on this
//              site to the next site of its chain (0 only on empty sites)
//   bit  4     label: the run holds monomer 0 of its chain
//   label clear: bits 16-31 run length, bits 5-15 zero
//   label set:   bits 5-31 chain id; the run length is in the chain record
//   0          empty site
// (Inside the specialised sweep kernels a labelled word is rewritten while its
// tile is on chip: bits 5-15 index a shared-memory label slot and bits 16-31
// hold the run length, so every on-chip word carries its count.)
// Chain record (4 x uint32 per chain): {global site of monomer 0's run,
//   length of that run, offset of monomer 0 inside it, unused}.
//
// A run is a maximal group of consecutive monomers of one ring on one site
// (the reference's stored length, cpupol/efpol_lib.c:132-207 with bond 0).
#pragma once
#include <stdint.h>
#include <stddef.h>

#define ELP_LBIT 16u
#define ELP_CSHIFT 16            // run length position
#define ELP_CUNIT (1u << 16)     // +1 monomer in a run
#define ELP_MAX_N 65536          // longest ring (run lengths fit 16 bits)
#define ELP_WALL 0xFFFFFFFFu
#define ELP_REC_WORDS 4

// Philox counter layout (c2 high bits select the stream).
#define ELP_STREAM_COLOUR 0x40000000u
#define ELP_STREAM_SHIFT 0x80000000u
#define ELP_STREAM_HEAD 0x20000000u    // monomer-0 moves of linear chains: ctr {t, d, k | HEAD, anchor}

#ifdef __CUDACC__
#define ELP_HD __host__ __device__ __forceinline__
#else
#define ELP_HD inline
#endif

// Bond code -> lattice vector components.
static ELP_HD int elp_bt(uint32_t b) { return (int)(b & 1) - (int)((b >> 3) & 1); }
static ELP_HD int elp_bu(uint32_t b) { return (int)((b >> 1) & 1) - (int)((b >> 3) & 1); }
static ELP_HD int elp_bv(uint32_t b) { return (int)((b >> 2) & 1) - (int)((b >> 3) & 1); }
static ELP_HD int elp_valid_bond(uint32_t a) { return a != 0 && a != 0x3 && a != 0xc && a != 0xf; }

// Domain geometry of one melt.  It is part of the trajectory's definition:
// the same melt with another geometry follows another (equally valid) chain.
struct elp_geometry {
    int L;          // cubic box edge
    int periodic;   // 1: the whole box is one periodic domain held on chip
    int tx, ty, tz; // tile edges (tiled); == L (periodic)
    int ncol;       // colour modulus n of (x + 2y + 3z) mod n; 2n substeps/step
};

// Shared-memory layout of one domain.
struct elp_smem_layout {
    int sx, sxy;        // row and plane strides in words
    int ox;             // index of local (0,0,0)
    int words;          // words of lattice storage
    int anchors;        // anchors per substep A
    int groups;         // A/4 = threads per domain
    size_t bytes;       // total dynamic shared memory
};

// Host helpers (elp_host.cpp).
int elp_pick_ncol(int L);
int elp_geometry_ok(const elp_geometry* g);
void elp_layout(const elp_geometry* g, elp_smem_layout* lay);
void elp_philox_host(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void elp_build_table(uint8_t tab[4096]);
int elp_get_npol(double density, int N, long sites);
// The grid of CreatePolymers (cpupol/efpol_init.c:239-283): chain p starts at
// (delta (p % nt), delta (p / nt / nv), (delta + 1) ((p / nt) % nv)).
// Returns 0, or 1 if it cannot hold P chains.
int elp_initial_grid(int L, int N, int P, int* delta, int* nt, int* nv);

