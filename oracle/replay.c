/*
 * replay.c -- TEST INFRASTRUCTURE ONLY (the bit-exact oracle of the GPU path).
 *
 * Host replay of the sweep schedule that the sm_100a kernels run.  The
 * reference's sequential efpol (cpupol/efpol_lib.c:122-207) cannot be matched
 * bit for bit by any parallel schedule, so the GPU path is checked against
 * this replay instead; the replay in turn applies exactly efpol's
 * single-monomer move (same table, cpupol/efpol_init.c:314-424) and is checked
 * statistically against efpol.
 *
 * State.  One uint32 word per lattice site (index t + L*(u + L*v)):
 *   bits 0-3  b_out: bond from the last monomer of the run on this site to
 *             the next site of the chain (never 0 on an occupied site)
 *   bit  4    label: the run holds monomer 0 of its chain
 *   unlabelled: bits 16-31 run length (bits 5-15 zero)
 *   labelled:   bits 5-31 chain id, run length in the chain record
 *   word 0    empty site
 * Per chain a record {site of monomer 0's run, its run length, offset of
 * monomer 0 inside that run}.
 *
 * Schedule of step t (all randomness from Philox4x32-10, key {seed, salt}):
 *   - tiled boxes: origin shift (st,su,sv) from ctr {t, 0, 0x80000000, 0};
 *     periodic boxes: the whole box is one domain, no shift.
 *   - every domain d runs 2n substeps k; colour c_k = bounded(word k&3 of
 *     ctr {t, d, (k>>2)|0x40000000, 0}, n); anchors are the domain sites with
 *     (x + 2y + 3z) mod n == c_k, enumerated a = j*R + row (row = y + Ty*z,
 *     x = ((c_k - 2y - 3z) mod n) + n*j).  Anchor a = g + q*(A/4) takes byte
 *     q of word k&3 of ctr {t, d, k>>2, g}: bit 0 = slot, bits 1-4 = option.
 *   - an anchor P moves the monomer whose predecessor sits on P: slot 0 the
 *     last monomer of P's run, slot 1 the first monomer of the next run.
 *     Move and reverse move share the anchor, all sites touched lie within
 *     one bond of P, and same-colour anchors are >= 3 bonds apart, so the
 *     substep is conflict-free and each substep kernel is symmetric.
 *
 * Linear chains (efpol built with POL_TYPE=POL_LIN): bond N-1 is the end
 * marker 0xf, stored as b_out of the chain's last run, and monomer 0 is the
 * first monomer of its run (offset 0).  The move above then covers the last
 * monomer (rows (u, 0xf) and (0, 0xf) of efpol's table); slot 1 at a last
 * run has no next run and is null.  Monomer 0 has no predecessor: it moves
 * about monomer 1 (efpol's rows (0xf, x)).  After its regular attempt, an
 * anchor holding a chain's monomer 0 draws word 0 of
 * ctr {t, d, k | 0x20000000, a}: bit 0 set -> one attempt with option bits
 * 1-4 in row (0xf, run length > 1 ? 0 : b_out): either monomer 0 leaves
 * its run to the empty site P - u (new bond u), or, alone on P, joins the
 * front of the next run.  All sites touched lie within one bond of P.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#define LBIT 16u
#define CSH 16

static uint8_t g_tab[4096];
static int g_tab_ready = 0;

static void tab_init(void)
{
    if (g_tab_ready) return;
    orc_table* T = (orc_table*)malloc(sizeof(orc_table));
    orc_build_table(T, ORC_SL_EQUAL, ORC_POL_RING);
    for (int i = 0; i < 4096; i++) g_tab[i] = (uint8_t)(T->trans[i] & 0xff);
    free(T);
    g_tab_ready = 1;
}

static inline uint32_t bounded(uint32_t w, uint32_t n) { return (uint32_t)(((uint64_t)w * n) >> 32); }

typedef struct dom {
    int L, periodic;
    int x0, y0, z0;      /* global coordinates of local (0,0,0) */
    int tx, ty, tz;
} dom;

static inline size_t dsite(const dom* D, int x, int y, int z)
{
    int L = D->L;
    int t = (D->x0 + x) % L, u = (D->y0 + y) % L, v = (D->z0 + z) % L;
    return (size_t)t + (size_t)L * ((size_t)u + (size_t)L * (size_t)v);
}

static inline int dnbr(const dom* D, int x, int y, int z, uint32_t b, int* nx, int* ny, int* nz)
{
    int dt, du, dv;
    orc_unit_vec(b, &dt, &du, &dv);
    x += dt; y += du; z += dv;
    if (D->periodic) {
        x = (x + D->L) % D->L; y = (y + D->L) % D->L; z = (z + D->L) % D->L;
    } else if (x < 0 || y < 0 || z < 0 || x >= D->tx || y >= D->ty || z >= D->tz) {
        return 0;
    }
    *nx = x; *ny = y; *nz = z;
    return 1;
}

static inline uint32_t w_count(const orc_replay* r, uint32_t w)
{
    return (w & LBIT) ? r->rec[4 * (size_t)(w >> 5) + 1] : (w >> CSH);
}

/* One anchored move attempt. Returns 1 if the move was applied. */
static int replay_op(orc_replay* r, const dom* D, int x, int y, int z, uint32_t s, uint32_t r4)
{
    uint32_t* lat = r->lat;
    size_t iP = dsite(D, x, y, z), iB = 0, iY;
    uint32_t wP = lat[iP];
    if (!wP) return 0;
    uint32_t bo = wP & 15, cP = w_count(r, wP);
    uint32_t src1, src2, wB = 0, cB = 0;
    int bx, by, bz, yx, yy, yz;
    if (s == 0) {
        if (cP < 2) return 0;
        src1 = 0;
        src2 = bo;
    } else {
        if (bo == 15) return 0;            /* last run of a linear chain: no next run */
        if (!dnbr(D, x, y, z, bo, &bx, &by, &bz)) return 0;
        iB = dsite(D, bx, by, bz);
        wB = lat[iB];
        cB = w_count(r, wB);
        src1 = bo;
        src2 = (cB >= 2) ? 0 : (wB & 15);
    }
    r->attempted++;
    uint32_t e = g_tab[(src1 << 8) | (src2 << 4) | r4];
    uint32_t d1 = e & 15, d2 = e >> 4;
    if (!d1 && !d2) return 0;
    iY = iP;
    if (d1) {
        if (!dnbr(D, x, y, z, d1, &yx, &yy, &yz)) return 0;
        iY = dsite(D, yx, yy, yz);
    }
    uint32_t wY = lat[iY];
    if (d1 && d2 && wY) return 0;            /* new site must be empty */
    uint32_t cN = d2 ? 0 : w_count(r, wY);  /* d2 == 0: m joins the next run */

    uint32_t nP_c = cP + (d1 == 0) - (src1 == 0);
    uint32_t wP2 = (d1 ? d1 : d2) | (nP_c << CSH);
    uint32_t wB2 = 0, wY2 = 0;
    if (s == 1 && src2 == 0) wB2 = (wB & 15) | ((cB - 1) << CSH);
    if (d1 && d2) wY2 = d2 | (1u << CSH);
    else if (!d2) wY2 = (wY & 15) | ((cN + 1) << CSH);

    /* monomer-0 label follows its monomer */
    int lab = -1, nl = -1;
    uint32_t chain = 0, noff = 0;
    if (wP & LBIT) { lab = 0; chain = wP >> 5; }
    else if (s == 1 && (wB & LBIT)) { lab = 1; chain = wB >> 5; }
    else if (!d2 && (wY & LBIT)) { lab = 2; chain = wY >> 5; }
    if (lab >= 0) {
        uint32_t off = r->rec[4 * (size_t)chain + 2];
        if (lab == 0) {
            nl = 0; noff = off;
            if (s == 0 && off == cP - 1) { nl = 2; noff = 0; }
        } else if (lab == 1) {
            if (src2 == 0 && off > 0) { nl = 1; noff = off - 1; }
            else { nl = d1 ? 2 : 0; noff = d1 ? 0 : nP_c - 1; }
        } else {
            nl = 2; noff = off + 1;
        }
        uint32_t* tgt = nl == 0 ? &wP2 : (nl == 1 ? &wB2 : &wY2);
        size_t site = nl == 0 ? iP : (nl == 1 ? iB : iY);
        r->rec[4 * (size_t)chain + 0] = (uint32_t)site;
        r->rec[4 * (size_t)chain + 1] = *tgt >> CSH;
        r->rec[4 * (size_t)chain + 2] = noff;
        *tgt = (*tgt & 15) | LBIT | (chain << 5);
    }
    lat[iP] = wP2;
    if (s == 1) lat[iB] = wB2;
    if (d1) lat[iY] = wY2;
    r->accepted++;
    return 1;
}

/* Monomer 0 of a linear chain, whose run sits on the anchor (see header). */
static int replay_head(orc_replay* r, const dom* D, int x, int y, int z, uint32_t r4)
{
    uint32_t* lat = r->lat;
    const size_t iP = dsite(D, x, y, z);
    const uint32_t wP = lat[iP];
    const uint32_t chain = wP >> 5, cP = r->rec[4 * (size_t)chain + 1], bo = wP & 15;
    const uint32_t e = g_tab[(15u << 8) | ((cP >= 2 ? 0u : bo) << 4) | r4];
    if (!e) return 0;
    const uint32_t d2 = e >> 4;
    int nx, ny, nz;
    if (cP >= 2) {
        /* monomer 0 leaves to P - d2, its bond to monomer 1 becoming d2 */
        if (!dnbr(D, x, y, z, (~d2) & 15u, &nx, &ny, &nz)) return 0;
        const size_t iY = dsite(D, nx, ny, nz);
        if (lat[iY]) return 0;
        lat[iP] = bo | ((cP - 1) << CSH);
        lat[iY] = d2 | LBIT | (chain << 5);
        r->rec[4 * (size_t)chain + 0] = (uint32_t)iY;
        r->rec[4 * (size_t)chain + 1] = 1;
    } else {
        /* alone on P: monomer 0 joins the front of the next run */
        if (!dnbr(D, x, y, z, bo, &nx, &ny, &nz)) return 0;
        const size_t iB = dsite(D, nx, ny, nz);
        const uint32_t wB = lat[iB];
        lat[iP] = 0;
        lat[iB] = (wB & 15) | LBIT | (chain << 5);
        r->rec[4 * (size_t)chain + 0] = (uint32_t)iB;
        r->rec[4 * (size_t)chain + 1] = (wB >> CSH) + 1;
    }
    r->rec[4 * (size_t)chain + 2] = 0;
    r->accepted++;
    return 1;
}

void orc_replay_set_linear(orc_replay* r, int linear) { r->linear = linear ? 1 : 0; }

void orc_replay_set_state(orc_replay* r, const uint32_t* lat, const uint32_t* rec, uint64_t step)
{
    const size_t S = (size_t)r->g.L * r->g.L * r->g.L;
    memcpy(r->lat, lat, S * sizeof(uint32_t));
    memcpy(r->rec, rec, 4 * (size_t)r->P * sizeof(uint32_t));
    r->step = step;
}

orc_replay* orc_replay_new(const orc_geom* g, int N, int P, uint32_t seed, uint32_t salt)
{
    tab_init();
    orc_replay* r = (orc_replay*)calloc(1, sizeof(orc_replay));
    r->g = *g;
    r->N = N; r->P = P; r->seed = seed; r->salt = salt;
    size_t S = (size_t)g->L * g->L * g->L;
    r->lat = (uint32_t*)calloc(S, sizeof(uint32_t));
    r->rec = (uint32_t*)calloc(4 * (size_t)P, sizeof(uint32_t));
    return r;
}

void orc_replay_free(orc_replay* r)
{
    if (!r) return;
    free(r->lat); free(r->rec); free(r);
}

static inline size_t gsite(int L, int t, int u, int v)
{
    t = ((t % L) + L) % L; u = ((u % L) + L) % L; v = ((v % L) + L) % L;
    return (size_t)t + (size_t)L * ((size_t)u + (size_t)L * (size_t)v);
}

/* Build site words from chains.  Returns 0, 3 (two runs on one site) or
 * 4 (invalid bond, ring not closed, or a chain on a single site). */
int orc_replay_load(orc_replay* r, const int32_t* start, const uint8_t* bonds)
{
    const int L = r->g.L, N = r->N;
    size_t S = (size_t)L * L * L;
    memset(r->lat, 0, S * sizeof(uint32_t));
    int* pt = (int*)malloc(sizeof(int) * 3 * (size_t)N);
    for (int p = 0; p < r->P; p++) {
        const uint8_t* b = bonds + (size_t)p * N;
        int t = start[3 * p], u = start[3 * p + 1], v = start[3 * p + 2];
        int nz = 0;
        if (r->linear && b[N - 1] != 15) { free(pt); return 4; }
        for (int m = 0; m < N; m++) {
            pt[3 * m] = t; pt[3 * m + 1] = u; pt[3 * m + 2] = v;
            if (b[m] && !orc_is_valid(b[m]) && !(r->linear && m == N - 1)) { free(pt); return 4; }
            int dt, du, dv;
            orc_unit_vec(b[m], &dt, &du, &dv);
            t += dt; u += du; v += dv;
            if (b[m]) nz++;
        }
        if (!r->linear && (gsite(L, t, u, v) != gsite(L, pt[0], pt[1], pt[2]) || nz < 2)) { free(pt); return 4; }
        /* runs start at monomers whose predecessor's bond is non-zero */
        int first = -1;
        for (int m = 0; m < N; m++) if (b[(m + N - 1) % N]) { first = m; break; }
        int m = first, done = 0;
        while (done < N) {
            int len = 1;
            while (b[(m + len - 1) % N] == 0) len++;
            size_t site = gsite(L, pt[3 * m], pt[3 * m + 1], pt[3 * m + 2]);
            if (r->lat[site]) { free(pt); return 3; }
            uint32_t bo = b[(m + len - 1) % N];
            int holds0 = ((0 - m + N) % N) < len;
            if (holds0) {
                r->lat[site] = bo | LBIT | ((uint32_t)p << 5);
                r->rec[4 * (size_t)p + 0] = (uint32_t)site;
                r->rec[4 * (size_t)p + 1] = (uint32_t)len;
                r->rec[4 * (size_t)p + 2] = (uint32_t)((0 - m + N) % N);
            } else {
                r->lat[site] = bo | ((uint32_t)len << CSH);
            }
            done += len;
            m = (m + len) % N;
        }
    }
    free(pt);
    return 0;
}

/* Walk every chain from monomer 0's run.  Returns 0 or 4 on any
 * inconsistency (chain not closing after exactly N monomers, bad bond). */
int orc_replay_export(const orc_replay* r, int32_t* start, uint8_t* bonds)
{
    const int L = r->g.L, N = r->N;
    for (int p = 0; p < r->P; p++) {
        uint32_t site = r->rec[4 * (size_t)p], cnt = r->rec[4 * (size_t)p + 1], off = r->rec[4 * (size_t)p + 2];
        uint32_t w = r->lat[site];
        if (!(w & LBIT) || (w >> 5) != (uint32_t)p || off >= cnt) return 4;
        start[3 * p] = (int32_t)(site % L);
        start[3 * p + 1] = (int32_t)((site / L) % L);
        start[3 * p + 2] = (int32_t)(site / ((uint32_t)L * L));
        uint8_t* b = bonds + (size_t)p * N;
        long i = 0;
        uint32_t here = cnt - off, cur = site;
        for (;;) {
            uint32_t bo = r->lat[cur] & 15;
            if (!(orc_is_valid(bo) || (r->linear && bo == 15)) || i + here > (long)N) return 4;
            for (uint32_t k = 0; k + 1 < here; k++) b[i++] = 0;
            b[i++] = (uint8_t)bo;
            if (bo == 15) break;      /* end of a linear chain */
            int dt, du, dv;
            orc_unit_vec(bo, &dt, &du, &dv);
            int t = (int)(cur % L), u = (int)((cur / L) % L), v = (int)(cur / ((uint32_t)L * L));
            cur = (uint32_t)gsite(L, t + dt, u + du, v + dv);
            uint32_t wn = r->lat[cur];
            if (!wn) return 4;
            if (cur == site) break;
            if (wn & LBIT) return 4;
            here = wn >> CSH;
        }
        if (i + (long)off != N) return 4;
        for (uint32_t k = 0; k < off; k++) b[i++] = 0;
    }
    return 0;
}

static void replay_step(orc_replay* r)
{
    const orc_geom* g = &r->g;
    const uint32_t t = (uint32_t)r->step;
    const uint32_t key[2] = {r->seed, r->salt};
    const int n = g->ncol;
    int tx = g->periodic ? g->L : g->tt;
    int ty = g->periodic ? g->L : g->tu;
    int tz = g->periodic ? g->L : g->tv;
    int st = 0, su = 0, sv = 0;
    if (!g->periodic) {
        uint32_t c[4] = {t, 0, 0x80000000u, 0}, o[4];
        orc_philox(c, key, o);
        st = (int)bounded(o[0], (uint32_t)tx);
        su = (int)bounded(o[1], (uint32_t)ty);
        sv = (int)bounded(o[2], (uint32_t)tz);
    }
    int nx = g->L / tx, ny = g->L / ty, nzt = g->L / tz;
    const int R = ty * tz, A = R * (tx / n), G = A / 4;
    uint32_t* words = (uint32_t*)malloc(sizeof(uint32_t) * 4 * (size_t)G);
    for (int d = 0; d < nx * ny * nzt; d++) {
        dom D;
        D.L = g->L; D.periodic = g->periodic;
        D.tx = tx; D.ty = ty; D.tz = tz;
        D.x0 = st + (d % nx) * tx;
        D.y0 = su + ((d / nx) % ny) * ty;
        D.z0 = sv + (d / nx / ny) * tz;
        uint32_t col[4] = {0, 0, 0, 0};
        for (int k = 0; k < 2 * n; k++) {
            if ((k & 3) == 0) {
                uint32_t c[4] = {t, (uint32_t)d, (uint32_t)(k >> 2) | 0x40000000u, 0};
                orc_philox(c, key, col);
                for (int gg = 0; gg < G; gg++) {
                    uint32_t c2[4] = {t, (uint32_t)d, (uint32_t)(k >> 2), (uint32_t)gg};
                    orc_philox(c2, key, words + 4 * (size_t)gg);
                }
            }
            int ck = (int)bounded(col[k & 3], (uint32_t)n);
            for (int gg = 0; gg < G; gg++) {
                uint32_t w = words[4 * (size_t)gg + (k & 3)];
                for (int q = 0; q < 4; q++) {
                    int a = gg + q * G;
                    int j = a / R, row = a % R;
                    int y = row % ty, z = row / ty;
                    int x = (((ck - 2 * y - 3 * z) % n) + n) % n + n * j;
                    uint32_t rb = (w >> (8 * q)) & 0xff;
                    replay_op(r, &D, x, y, z, rb & 1, (rb >> 1) & 15);
                    if (r->linear && (r->lat[dsite(&D, x, y, z)] & LBIT)) {
                        uint32_t hc[4] = {t, (uint32_t)d, (uint32_t)k | 0x20000000u, (uint32_t)a}, hw[4];
                        orc_philox(hc, key, hw);
                        if (hw[0] & 1) replay_head(r, &D, x, y, z, (hw[0] >> 1) & 15);
                    }
                }
            }
        }
    }
    free(words);
}

void orc_replay_steps(orc_replay* r, long nsteps)
{
    for (long i = 0; i < nsteps; i++) {
        replay_step(r);
        r->step++;
    }
}
