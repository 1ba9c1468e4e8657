/*
 * efpol_port.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU restatement of the reference's ELP algorithm, written from the
 * reference's behaviour, used to pin golden vectors and as the statistical
 * and timing baseline.  Every function names the reference code it follows.
 *
 * The restatement must reproduce the reference efpol bit for bit: identical
 * transition table, identical t=0 configuration, and -- because it consumes
 * the Tausworthe stream in the same order -- identical trajectories.  The
 * tests check all three against fixtures produced by the reference itself.
 */
#include "oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- FCC unit algebra: cpupol/efpol_lib.c:21-48, 83-93 ------------------
 * A bond is a 4-bit code over the basis (t, u, v, w) with w = -(t+u+v).
 * Codes 0, 0x3, 0xc and 0xf are not nearest-neighbour bonds. */
int orc_is_valid(uint32_t a) { return a != 0 && a != 0x3 && a != 0xc && a != 0xf; }

/* Sum of two bonds if it is itself a bond (ValidateAddUnitVectors). */
int orc_add_units(uint32_t a, uint32_t b, uint32_t* c)
{
    if ((a | b) != 0xf && (a & b)) return 0;
    uint32_t r = ((a | b) == 0xf) ? (a & b) : (a | b);
    *c = r;
    return orc_is_valid(r);
}

void orc_unit_vec(uint32_t u, int* dt, int* du, int* dv)
{
    int w = (int)((u >> 3) & 1);
    *dt = (int)(u & 1) - w;
    *du = (int)((u >> 1) & 1) - w;
    *dv = (int)((u >> 2) & 1) - w;
}

/* GetNPol, cpupol/efpol_lib.c:50-56 */
int orc_get_npol(double density, int N, long sites)
{
    double d = density * (double)sites / (double)N;
    return (int)(d + 0.5);
}

/* ---- transition table: cpupol/efpol_init.c:285-424 ----------------------
 * For every (src1, src2) bond pair around a monomer the table lists 16
 * options dst1 | dst2<<4 | move<<8; a 4-bit random number picks one. */
static void tab_add(orc_table* T, uint32_t s1, uint32_t s2, uint32_t d1, uint32_t d2)
{
    int id = 256 * (int)s1 + 16 * (int)s2 + T->ntrans[16 * s1 + s2];
    if (id >= 4096) return; /* cannot happen for the three models */
    T->trans[id] = d1 | (d2 << 4);
    if (d1 || d2) {
        uint32_t mv = 0;
        int ok = (d1 != 0xf) ? orc_add_units(d1, (~s1) & 0xf, &mv)
                             : orc_add_units(s2, (~d2) & 0xf, &mv);
        if (!ok) { fprintf(stderr, "oracle: bad transition %x,%x->%x,%x\n", s1, s2, d1, d2); abort(); }
        T->trans[id] |= mv << 8;
    }
    T->rem_occ[id] = (s1 && s2) ? 1 : 0;
    T->add_occ[id] = (d1 && d2) ? 1 : 0;
    T->ntrans[16 * s1 + s2]++;
}

static int vec_sum_zero(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    /* a + b - c - d == 0 as lattice vectors */
    int at, au, av, bt, bu, bv, ct, cu, cv, dt, du, dv;
    orc_unit_vec(a, &at, &au, &av); orc_unit_vec(b, &bt, &bu, &bv);
    orc_unit_vec(c, &ct, &cu, &cv); orc_unit_vec(d, &dt, &du, &dv);
    return at + bt - ct - dt == 0 && au + bu - cu - du == 0 && av + bv - cv - dv == 0;
}

void orc_build_table(orc_table* T, int model, int pol_type)
{
    memset(T, 0, sizeof(*T));
    (void)pol_type;
    /* kink <-> stored length: efpol_init.c:320-337 */
    for (uint32_t a = 1; a < 0xf; a++) {
        if (!orc_is_valid(a)) continue;
        for (uint32_t b = a + 1; b < 0xf; b++) {
            uint32_t r;
            if (!orc_is_valid(b) || !orc_add_units(a, b, &r)) continue;
            tab_add(T, a, b, r, 0); tab_add(T, a, b, 0, r);
            tab_add(T, b, a, r, 0); tab_add(T, b, a, 0, r);
            tab_add(T, r, 0, a, b); tab_add(T, r, 0, b, a);
            tab_add(T, 0, r, a, b); tab_add(T, 0, r, b, a);
        }
    }
    /* stored-length hop along a bond, 4 copies each: efpol_init.c:339-345 */
    for (uint32_t b = 1; b < 0xf; b++) {
        if (!orc_is_valid(b)) continue;
        for (int i = 0; i < 4; i++) { tab_add(T, 0, b, b, 0); tab_add(T, b, 0, 0, b); }
    }
    /* crankshaft / hairpin rotations: efpol_init.c:347-376 */
    for (uint32_t u1 = 1; u1 < 0xf; u1++) {
        if (!orc_is_valid(u1)) continue;
        for (uint32_t u2 = 1; u2 < 0xf; u2++) {
            uint32_t r;
            if (!orc_is_valid(u2) || !orc_add_units(u1, (~u2) & 0xf, &r)) continue;
            for (uint32_t u3 = 1; u3 < 0xf; u3++) {
                if (!orc_is_valid(u3)) continue;
                if (model == ORC_SL_QUAD && orc_add_units(u1, u3, &r)) continue;
                for (uint32_t u4 = 1; u4 < 0xf; u4++) {
                    if (!orc_is_valid(u4) || !vec_sum_zero(u1, u3, u2, u4)) continue;
                    tab_add(T, u1, u3, u2, u4); tab_add(T, u1, u3, u2, u4);
                    if (model == ORC_SL_EQUAL && orc_add_units(u1, u3, &r))
                        for (int i = 0; i < 4; i++) tab_add(T, u1, u3, u2, u4);
                }
            }
        }
    }
    /* Rows holding exactly 2, 4 or 8 entries are repeated; the three tests run
     * one after the other on the growing row, so 2 -> 4 -> 8 -> 16
     * (efpol_init.c:378-400). */
    for (int row = 0; row < 256; row++) {
        for (int want = 2; want <= 8; want *= 2) {
            if (T->ntrans[row] != want) continue;
            for (int i = 0; i < want; i++) {
                uint32_t e = T->trans[row * 16 + i];
                tab_add(T, (uint32_t)row / 16, (uint32_t)row % 16, e & 0xf, (e >> 4) & 0xf);
            }
        }
    }
    /* linear-chain end moves: efpol_init.c:402-416 */
    for (uint32_t a = 0; a < 0xf; a++) {
        if (!orc_is_valid(a)) continue;
        for (int i = 0; i < model; i++) { tab_add(T, a, 0xf, 0x0, 0xf); tab_add(T, 0xf, a, 0xf, 0x0); }
        tab_add(T, 0x0, 0xf, a, 0xf);
        tab_add(T, 0xf, 0x0, 0xf, a);
    }
    /* pad every row with null moves to 16 entries: efpol_init.c:417-421 */
    for (int row = 0; row < 256; row++)
        while (T->ntrans[row] < 16) tab_add(T, (uint32_t)row / 16, (uint32_t)row % 16, 0, 0);
}

/* ---- Tausworthe generator: util/rng.h:10-35 ------------------------------ */
static uint32_t taus(uint32_t* s)
{
    uint32_t b;
    b = ((s[0] << 6) ^ s[0]) >> 13;  s[0] = ((s[0] & 4294967294u) << 18) ^ b;
    b = ((s[1] << 2) ^ s[1]) >> 27;  s[1] = ((s[1] & 4294967288u) << 2) ^ b;
    b = ((s[2] << 13) ^ s[2]) >> 21; s[2] = ((s[2] & 4294967280u) << 7) ^ b;
    b = ((s[3] << 3) ^ s[3]) >> 12;  s[3] = ((s[3] & 4294967168u) << 13) ^ b;
    return s[0] ^ s[1] ^ s[2] ^ s[3];
}
static double taus_unit(uint32_t* s) { return 2.3283064365386962890625E-10 * (double)taus(s); }

/* ---- state ---------------------------------------------------------------- */
static inline uint32_t bond_get(const orc_efpol* s, int mono, int pol)
{
    return (s->unit[(size_t)mono * s->ints_per_mono + pol / 8] >> (4 * (pol % 8))) & 0xf;
}
static inline void bond_set(orc_efpol* s, int mono, int pol, uint32_t b)
{
    uint32_t* w = &s->unit[(size_t)mono * s->ints_per_mono + pol / 8];
    *w = (*w & ~(0xfu << (4 * (pol % 8)))) | (b << (4 * (pol % 8)));
}
static inline uint32_t add_bond(const orc_efpol* s, uint32_t coor, uint32_t b)
{
    int L = s->L, dt, du, dv;
    orc_unit_vec(b, &dt, &du, &dv);
    int t = (int)(coor % L), u = (int)((coor / L) % L), v = (int)(coor / ((uint32_t)L * L));
    t = (t + dt + L) % L; u = (u + du + L) % L; v = (v + dv + L) % L;
    return (uint32_t)(t + L * (u + L * v));
}
static inline int occ_get(const uint32_t* o, uint32_t c) { return (o[c >> 5] >> (c & 31)) & 1; }
static inline void occ_set(uint32_t* o, uint32_t c) { o[c >> 5] |= 1u << (c & 31); }
static inline void occ_clr(uint32_t* o, uint32_t c) { o[c >> 5] &= ~(1u << (c & 31)); }

/* CSInit + ConfigInit (efpol_init.c:55-78, 426-433; util/rng.h:26-31) */
orc_efpol* orc_efpol_new(int L, int N, int P, int pol_type, int model, uint32_t seed)
{
    orc_efpol* s = (orc_efpol*)calloc(1, sizeof(orc_efpol));
    s->L = L; s->N = N; s->P = P; s->pol_type = pol_type;
    s->ints_per_mono = (P + 7) / 8;
    size_t sites = (size_t)L * L * L;
    s->coor = (uint32_t*)calloc((size_t)N * P, sizeof(uint32_t));
    s->unit = (uint32_t*)calloc((size_t)N * s->ints_per_mono, sizeof(uint32_t));
    s->occ = (uint32_t*)calloc(sites / 32 + 1, sizeof(uint32_t));
    s->rng[0] = seed; s->rng[1] = seed ^ 0xa741f123u;
    s->rng[2] = seed ^ 0x213910abu; s->rng[3] = seed ^ 0xcd123e14u;
    orc_build_table(&s->tab, model, pol_type);
    return s;
}

void orc_efpol_free(orc_efpol* s)
{
    if (!s) return;
    free(s->coor); free(s->unit); free(s->occ); free(s);
}

/* CreatePolymers, efpol_init.c:239-283: chains start on a delta-spaced grid,
 * each as two sites: monomer 0 alone, then bond +v to the other N-1. */
void orc_efpol_create(orc_efpol* s)
{
    int L = s->L, delta;
    for (delta = 1; delta < L; delta++) {
        long ntot = (long)(L / delta) * (L / delta) * (L / (delta + 1));
        if (ntot < s->P) { delta--; break; }
    }
    int nt = L / delta, nv = L / (delta + 1);
    for (int p = 0; p < s->P; p++) {
        int t = delta * (p % nt);
        int v = (delta + 1) * ((p / nt) % nv);
        int u = delta * (p / nt / nv);
        uint32_t a = (uint32_t)(t + L * (u + L * v));
        uint32_t b = (uint32_t)(t + L * (u + L * (v + 1)));
        s->coor[p] = a;
        bond_set(s, 0, p, 0x4);
        occ_set(s->occ, a); occ_set(s->occ, b);
        for (int m = 1; m < s->N; m++) s->coor[(size_t)m * s->P + p] = b;
        bond_set(s, s->N - 1, p, s->pol_type == ORC_POL_LIN ? 0xf : 0xb);
    }
}

/* DoStep, efpol_lib.c:132-207: one monomer index for a block of 8 chains,
 * one 4-bit option per chain from a shared 32-bit draw. */
static int efpol_dostep(orc_efpol* s)
{
    const int N = s->N, P = s->P;
    int mono = (int)(taus_unit(s->rng) * N);
    int prev = (s->pol_type == ORC_POL_LIN) ? (mono == 0 ? N - 1 : mono - 1) : (mono - 1 + N) % N;
    int nblk = (P - 1) / 8 + 1;
    int p0 = (int)(taus_unit(s->rng) * nblk) * 8;
    int p1 = p0 + 8 < P ? p0 + 8 : P;
    uint32_t ropt = 0;
    int changed = 0;
    for (int p = p0; p < p1; p++) {
        int sh = (p - p0) % 8;
        if (sh == 0) ropt = taus(s->rng);
        uint32_t s1 = bond_get(s, prev, p), s2 = bond_get(s, mono, p);
        int opt = (int)(s1 * 256 + s2 * 16 + ((ropt >> (4 * sh)) & 0xf));
        uint32_t e = s->tab.trans[opt];
        uint32_t d1 = e & 0xf, d2 = (e >> 4) & 0xf, mv = e >> 8;
        if (!d1 && !d2) continue;
        uint32_t old = s->coor[(size_t)mono * P + p];
        uint32_t nw = add_bond(s, old, mv);
        if (s->tab.add_occ[opt]) {
            if (occ_get(s->occ, nw)) continue;
            occ_set(s->occ, nw);
        }
        if (s->tab.rem_occ[opt]) occ_clr(s->occ, old);
        s->coor[(size_t)mono * P + p] = nw;
        bond_set(s, prev, p, d1);
        bond_set(s, mono, p, d2);
        changed++;
    }
    return changed;
}

/* DoMCStep, efpol_lib.c:122-129: interval*N*ceil(P/8) DoSteps */
long orc_efpol_mcstep(orc_efpol* s, long ntime)
{
    long nsmall = ntime * s->N * ((s->P - 1) / 8 + 1), acc = 0;
    for (long j = 0; j < nsmall; j++) acc += efpol_dostep(s);
    return acc;
}

/* CheckIntegrity, efpol_io.c:158-211: 0 ok, 2 coordinate/bond mismatch,
 * 3 double occupancy, 4 invalid bond, broken ring or stale occupancy. */
int orc_efpol_check(const orc_efpol* s)
{
    size_t sites = (size_t)s->L * s->L * s->L;
    uint32_t* chk = (uint32_t*)calloc(sites / 32 + 1, sizeof(uint32_t));
    int rc = 0;
    for (int p = 0; p < s->P && !rc; p++) {
        uint32_t c = s->coor[p];
        for (int m = 0; m < s->N; m++) {
            if (c != s->coor[(size_t)m * s->P + p]) { rc = 2; break; }
            uint32_t b = bond_get(s, m, p);
            int lin_end = (s->pol_type == ORC_POL_LIN && b == 0xf && m == s->N - 1);
            if (!orc_is_valid(b) && b != 0 && !lin_end) { rc = 4; break; }
            if (b && occ_get(chk, c) && !(s->pol_type == ORC_POL_RING && m == s->N - 1)) { rc = 3; break; }
            if (b) occ_set(chk, c);
            if (!lin_end) c = add_bond(s, c, b);
        }
        if (!rc && s->pol_type == ORC_POL_RING && c != s->coor[p]) rc = 4;
    }
    if (!rc) {
        for (size_t i = 0; i < sites / 32 + 1; i++)
            if (chk[i] != s->occ[i]) { rc = 4; break; }
    }
    free(chk);
    return rc;
}

/* WriteLatticeFile / WritePolymer, efpol_io.c:50-77 */
long orc_efpol_write_tuv(const orc_efpol* s, char* buf, long cap)
{
    long n = 0;
    int L = s->L;
#define EMIT(...)                                                              \
    do {                                                                       \
        int k_ = snprintf(buf + n, (size_t)(cap > n ? cap - n : 0), __VA_ARGS__); \
        if (k_ < 0 || n + k_ >= cap) return -1;                                \
        n += k_;                                                               \
    } while (0)
    EMIT("LT= %i\nLU= %i\nLV= %i\nnp= %i\nmaxPolLength= %i\n", L, L, L, s->P, s->N);
    for (int p = 0; p < s->P; p++) {
        uint32_t c = s->coor[p];
        EMIT("len= %i\n%u  %u  %u\t", s->N, c % L, (c / L) % L, c / ((uint32_t)L * L));
        if (n + s->N + 1 >= cap) return -1;
        for (int m = 0; m < s->N; m++) buf[n++] = "0123456789abcdef"[bond_get(s, m, p)];
        buf[n++] = '\n';
    }
    buf[n] = '\0';
#undef EMIT
    return n;
}

/* ReadLatticeFile, efpol_io.c:3-47 */
int orc_efpol_read_tuv(orc_efpol* s, const char* text)
{
    int lt, lu, lv, np, ml, off = 0, k = 0;
    if (sscanf(text, "%*s %d %*s %d %*s %d %*s %d %*s %d%n", &lt, &lu, &lv, &np, &ml, &off) != 5) return 10;
    if (lt != s->L || lu != s->L || lv != s->L || np != s->P || ml != s->N) return 10;
    size_t sites = (size_t)s->L * s->L * s->L;
    memset(s->occ, 0, (sites / 32 + 1) * sizeof(uint32_t));
    memset(s->unit, 0, (size_t)s->N * s->ints_per_mono * sizeof(uint32_t));
    const char* q = text + off;
    char* str = (char*)malloc((size_t)s->N + 2);
    for (int p = 0; p < s->P; p++) {
        int len;
        unsigned t, u, v;
        if (sscanf(q, "%*s %d %u %u %u%n", &len, &t, &u, &v, &k) != 4 || len != s->N) { free(str); return 11; }
        q += k;
        while (*q == ' ' || *q == '\t' || *q == '\n') q++;
        int m = 0;
        while (q[m] && q[m] != '\n' && m <= s->N) { str[m] = q[m]; m++; }
        if (m != s->N) { free(str); return 11; }
        q += m;
        uint32_t c = (uint32_t)(t + (uint32_t)s->L * (u + (uint32_t)s->L * v));
        for (int i = 0; i < s->N; i++) {
            char ch = str[i];
            uint32_t b = (uint32_t)(ch <= '9' ? ch - '0' : ch - 'a' + 10);
            s->coor[(size_t)i * s->P + p] = c;
            occ_set(s->occ, c);
            bond_set(s, i, p, b);
            if (b != 0xf) c = add_bond(s, c, b);
        }
    }
    free(str);
    return 0;
}

void orc_efpol_export(const orc_efpol* s, int32_t* start, uint8_t* bonds)
{
    int L = s->L;
    for (int p = 0; p < s->P; p++) {
        uint32_t c = s->coor[p];
        start[3 * p] = (int32_t)(c % L);
        start[3 * p + 1] = (int32_t)((c / L) % L);
        start[3 * p + 2] = (int32_t)(c / ((uint32_t)L * L));
        for (int m = 0; m < s->N; m++) bonds[(size_t)p * s->N + m] = (uint8_t)bond_get(s, m, p);
    }
}
