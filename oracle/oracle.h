/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference ELP algorithm (efpol) and a host replay of
 * this project's GPU sweep schedule.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this code, and only as a checker or a
 * baseline; the product library never links it.
 *
 * Parity of the efpol restatement is pinned against the reference itself:
 * tests/golden/ holds the reference's transition table and trajectories
 * produced by the reference's own efpol built from its sources (oracle/Makefile,
 * target `ref`; generator tests/golden/make_golden.py).
 */
#ifndef ELP_ORACLE_H
#define ELP_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- efpol restatement (cpupol/efpol_*.c) ---------------- */

#define ORC_POL_RING 1
#define ORC_POL_LIN  2
#define ORC_SL_EQUAL 1
#define ORC_SL_DOUBLE 2
#define ORC_SL_QUAD 4

typedef struct orc_table {
    uint32_t trans[4096];   /* dst1 | dst2<<4 | move<<8  (cpupol/efpol.h:50) */
    int32_t  add_occ[4096];
    int32_t  rem_occ[4096];
    int32_t  ntrans[256];
} orc_table;

typedef struct orc_efpol {
    int L, N, P, pol_type;
    int ints_per_mono;        /* ceil(P/8) */
    uint32_t* coor;           /* [mono][pol]: t + L*u + L*L*v          */
    uint32_t* unit;           /* [mono][pol/8]: 4-bit bonds, 8 chains/word */
    uint32_t* occ;            /* occupancy bits, one per site           */
    uint32_t rng[4];          /* util/rng.h Tausworthe state           */
    orc_table tab;
} orc_efpol;

int  orc_is_valid(uint32_t a);
int  orc_add_units(uint32_t a, uint32_t b, uint32_t* c);
void orc_unit_vec(uint32_t u, int* dt, int* du, int* dv);
int  orc_get_npol(double density, int N, long sites);
void orc_build_table(orc_table* tab, int model, int pol_type);

orc_efpol* orc_efpol_new(int L, int N, int P, int pol_type, int model, uint32_t seed);
void orc_efpol_free(orc_efpol* s);
void orc_efpol_create(orc_efpol* s);            /* CreatePolymers */
long orc_efpol_mcstep(orc_efpol* s, long ntime); /* DoMCStep       */
int  orc_efpol_check(const orc_efpol* s);        /* CheckIntegrity, 0 = ok */
/* TUV text (cpupol/efpol_io.c:50-77).  Returns bytes written, or -1. */
long orc_efpol_write_tuv(const orc_efpol* s, char* buf, long cap);
int  orc_efpol_read_tuv(orc_efpol* s, const char* text);
/* start[3*P] (t,u,v of monomer 0) and bonds[P*N] */
void orc_efpol_export(const orc_efpol* s, int32_t* start, uint8_t* bonds);

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ---------------- */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---------------- replay of the GPU sweep schedule ---------------- */

typedef struct orc_geom {
    int L;           /* box edge (cubic)                                  */
    int periodic;    /* 1: whole box is one periodic domain               */
    int tt, tu, tv;  /* tile edge lengths (tiled mode)                    */
    int ncol;        /* colour modulus n; 2n substeps per step            */
} orc_geom;

typedef struct orc_replay {
    orc_geom g;
    int N, P;
    uint32_t seed, salt;
    uint64_t step;            /* absolute steps done */
    uint32_t* lat;            /* L^3 site words */
    uint32_t* rec;            /* 4 words per chain: site, count, offset, 0 */
    uint64_t accepted, attempted;
    int linear;               /* 1: linear chains (last run's b_out is 0xf) */
} orc_replay;

orc_replay* orc_replay_new(const orc_geom* g, int N, int P, uint32_t seed, uint32_t salt);
void orc_replay_free(orc_replay* r);
/* Build site words from chains: start[3*P], bonds[P*N]. 0 = ok. */
int  orc_replay_load(orc_replay* r, const int32_t* start, const uint8_t* bonds);
/* Walk chains back out of the site words. 0 = ok, else integrity code. */
int  orc_replay_export(const orc_replay* r, int32_t* start, uint8_t* bonds);
void orc_replay_steps(orc_replay* r, long nsteps);
/* Linear chains (set before load). */
void orc_replay_set_linear(orc_replay* r, int linear);
/* Take a state as it stands (site words L^3, records 4*P, in the layout
 * above) at absolute step `step`: e.g. a melt the GPU has relaxed. */
void orc_replay_set_state(orc_replay* r, const uint32_t* lat, const uint32_t* rec, uint64_t step);

#ifdef __cplusplus
}
#endif
#endif
