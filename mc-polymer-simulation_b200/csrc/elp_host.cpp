// elp_host.cpp -- host-side core of the ELP engine: geometry policy,
// shared-memory layout, the transition table, the initial melt and the
// conversion between chain form (start site + bond string, the TUV content)
// and site words.
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "elp_internal.h"

// ---- colouring -------------------------------------------------------------
// Same-colour sites (x + 2y + 3z = c mod n) must be at least three bonds
// apart so that two anchors' radius-1 footprints never meet: no sum of two
// bonds (other than 0) may have colour 0.
static int colour_ok(int n)
{
    if (n < 13) return 0;
    for (uint32_t a = 0; a < 16; a++) {
        if (a && !elp_valid_bond(a)) continue;
        for (uint32_t b = 0; b < 16; b++) {
            if (b && !elp_valid_bond(b)) continue;
            int dt = elp_bt(a) + elp_bt(b), du = elp_bu(a) + elp_bu(b), dv = elp_bv(a) + elp_bv(b);
            if (!dt && !du && !dv) continue;
            int c = ((dt + 2 * du + 3 * dv) % n + n) % n;
            if (c == 0) return 0;
        }
    }
    return 1;
}

// Smallest valid colour modulus that divides m (16 preferred).
int elp_pick_ncol(int m)
{
    if (m % 16 == 0) return 16;
    for (int n = 13; n <= m; n++)
        if (m % n == 0 && colour_ok(n)) return n;
    return 0;
}

int elp_geometry_ok(const elp_geometry* g)
{
    if (!g || g->L < 5 || g->L > 1024) return 0;
    if (!colour_ok(g->ncol)) return 0;
    if (g->periodic) {
        if (g->tx != g->L || g->ty != g->L || g->tz != g->L) return 0;
        if (g->L % g->ncol) return 0;
    } else {
        if (g->tx < 3 || g->ty < 3 || g->tz < 3) return 0;
        if (g->L % g->tx || g->L % g->ty || g->L % g->tz) return 0;
        if (g->tx % g->ncol) return 0;
    }
    long R = (long)g->ty * g->tz;
    long A = R * (g->tx / g->ncol);
    if (A % 4) return 0;
    if (A / 4 > 1024) return 0;
    elp_smem_layout lay;
    elp_layout(g, &lay);
    if (lay.bytes > 227u * 1024u) return 0;
    return 1;
}

// Worst shared-memory bank multiplicity of the first anchor load of a warp,
// over all colours and warps.
static int bank_cost(const elp_geometry* g, int ox, int sx, int sxy, bool permuted)
{
    int n = g->ncol, ty = g->ty, tz = g->tz;
    long R = (long)ty * tz, A = R * (g->tx / n), G = A / 4;
    int worst = 1;
    for (int c = 0; c < n; c++) {
        for (long w0 = 0; w0 < G && w0 < 32 * 8; w0 += 32) {
            int cnt[32] = {0};
            for (long g0 = w0; g0 < w0 + 32 && g0 < G; g0++) {
                long j = g0 / R, row = g0 % R;
                if (permuted) {  // lane -> row of an 8 x 4 block of rows
                    const long lane = row & 31, w = row >> 5;
                    row = (lane & 7) + 8 * (w % (ty / 8)) + (long)ty * ((lane >> 3) + 4 * (w / (ty / 8)));
                }
                int y = (int)(row % ty), z = (int)(row / ty);
                int x = (((c - 2 * y - 3 * z) % n) + n) % n + n * (int)j;
                long idx = ox + x + (long)sx * y + (long)sxy * z;
                int b = (int)(idx & 31);
                if (++cnt[b] > worst) worst = cnt[b];
            }
        }
    }
    return worst;
}

// Whole box: rows of L words (padded for banks).  Tiles: each row holds the
// 16-byte aligned span of TX + 4 words that the tile copy fetches (the tile
// at offset x0 mod 4 in it) and one halo word before it, so the row stride is
// a multiple of 4 words and at least TX + 5; rows y = -1, TY and planes
// z = -1, TZ are halo.  The specialised kernels hand out anchors to a warp's
// threads from an 8 x 4 block of (y, z) rows where the tile allows
// (`permuted`), which the bank score follows.
static void layout_search(const elp_geometry* g, elp_smem_layout* lay)
{
    const int per = g->periodic;
    const long A = (long)g->ty * g->tz * (g->tx / g->ncol), R = (long)g->ty * g->tz;
    // threads own one or two anchors in the tiled shapes: AT = A or A / 2
    const bool permuted = !per && g->ty % 8 == 0 && g->tz % 4 == 0 && (A % R == 0) && ((A / 2) % R == 0 || A == R);
    int best_sx = 0, best_sxy = 0, best = 1 << 30;
    const int sx0 = per ? g->tx : (g->tx + 5 + 3) & ~3;
    for (int px = 0; px < 8; px++) {
        int sx = per ? sx0 + px : sx0 + 4 * (px & 1);
        if (!per && px > 1) break;
        for (int pz = 0; pz < 32; pz += 1) {
            int sxy = per ? sx * g->ty + pz : sx * (g->ty + 2) + 4 * pz;
            int ox = per ? 0 : sx + sxy + 4;
            int cost = bank_cost(g, ox, sx, sxy, permuted) * 64 + px + pz;  // prefer small padding
            if (cost < best) { best = cost; best_sx = sx; best_sxy = sxy; }
        }
    }
    lay->sx = best_sx;
    lay->sxy = best_sxy;
    lay->ox = per ? 0 : best_sx + best_sxy + 4;
    lay->words = per ? best_sxy * g->tz
                     : ((lay->ox + best_sx * g->ty + best_sxy * g->tz + g->tx + 4 + 3) & ~3);
    lay->anchors = (int)A;
    lay->groups = lay->anchors / 4;
    lay->bytes = (size_t)lay->words * 4 + 4096 + 27 * 16 * 4 + 64 * 4;
}

// The padding search scores hundreds of candidate strides (milliseconds); a
// geometry's layout is computed once per process and reused (every job
// submitted to the serving loop resolves its geometry through here).
void elp_layout(const elp_geometry* g, elp_smem_layout* lay)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, int, int, int>, elp_smem_layout> memo;
    const auto key = std::make_tuple(g->L, g->periodic, g->tx, g->ty, g->tz, g->ncol);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = memo.find(key);
        if (it != memo.end()) {
            *lay = it->second;
            return;
        }
    }
    layout_search(g, lay);
    std::lock_guard<std::mutex> lk(mu);
    memo.emplace(key, *lay);
}

// ---- Philox4x32-10 (host copy; Salmon et al. SC'11) --------------------------
void elp_philox_host(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1; c3 = (uint32_t)p0; c0 = n0; c2 = n2;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// ---- transition table (sl_equal, rings): cpupol/efpol_init.c:285-424 --------
// Built by the same steps as the reference so that the 16 options of every
// (b_{m-1}, b_m) row, with their multiplicities and order, are identical.
namespace {
struct TableBuilder {
    uint32_t e[4096];
    int cnt[256];
    void add(uint32_t s1, uint32_t s2, uint32_t d1, uint32_t d2)
    {
        int id = 256 * (int)s1 + 16 * (int)s2 + cnt[16 * s1 + s2];
        if (id < 4096) e[id] = d1 | (d2 << 4);
        cnt[16 * s1 + s2]++;
    }
};
int sum_bond(uint32_t a, uint32_t b, uint32_t* c)
{
    if ((a | b) != 0xf && (a & b)) return 0;
    *c = ((a | b) == 0xf) ? (a & b) : (a | b);
    return elp_valid_bond(*c);
}
}  // namespace

void elp_build_table(uint8_t tab[4096])
{
    TableBuilder T;
    memset(&T, 0, sizeof(T));
    for (uint32_t a = 1; a < 0xf; a++) {
        if (!elp_valid_bond(a)) continue;
        for (uint32_t b = a + 1; b < 0xf; b++) {
            uint32_t r;
            if (!elp_valid_bond(b) || !sum_bond(a, b, &r)) continue;
            T.add(a, b, r, 0); T.add(a, b, 0, r); T.add(b, a, r, 0); T.add(b, a, 0, r);
            T.add(r, 0, a, b); T.add(r, 0, b, a); T.add(0, r, a, b); T.add(0, r, b, a);
        }
    }
    for (uint32_t b = 1; b < 0xf; b++) {
        if (!elp_valid_bond(b)) continue;
        for (int i = 0; i < 4; i++) { T.add(0, b, b, 0); T.add(b, 0, 0, b); }
    }
    for (uint32_t u1 = 1; u1 < 0xf; u1++) {
        if (!elp_valid_bond(u1)) continue;
        for (uint32_t u2 = 1; u2 < 0xf; u2++) {
            uint32_t r;
            if (!elp_valid_bond(u2) || !sum_bond(u1, (~u2) & 0xf, &r)) continue;
            for (uint32_t u3 = 1; u3 < 0xf; u3++) {
                if (!elp_valid_bond(u3)) continue;
                int kink = sum_bond(u1, u3, &r);
                for (uint32_t u4 = 1; u4 < 0xf; u4++) {
                    if (!elp_valid_bond(u4)) continue;
                    if (elp_bt(u1) + elp_bt(u3) != elp_bt(u2) + elp_bt(u4)) continue;
                    if (elp_bu(u1) + elp_bu(u3) != elp_bu(u2) + elp_bu(u4)) continue;
                    if (elp_bv(u1) + elp_bv(u3) != elp_bv(u2) + elp_bv(u4)) continue;
                    int copies = kink ? 6 : 2;
                    for (int i = 0; i < copies; i++) T.add(u1, u3, u2, u4);
                }
            }
        }
    }
    for (int row = 0; row < 256; row++)
        for (int want = 2; want <= 8; want *= 2)
            if (T.cnt[row] == want)
                for (int i = 0; i < want; i++) {
                    uint32_t v = T.e[row * 16 + i];
                    T.add((uint32_t)row / 16, (uint32_t)row % 16, v & 0xf, (v >> 4) & 0xf);
                }
    for (uint32_t a = 0; a < 0xf; a++) {
        if (!elp_valid_bond(a)) continue;
        T.add(a, 0xf, 0x0, 0xf); T.add(0xf, a, 0xf, 0x0);  // linear-chain ends (sl_equal: once)
        T.add(0x0, 0xf, a, 0xf); T.add(0xf, 0x0, 0xf, a);
    }
    for (int row = 0; row < 256; row++)
        while (T.cnt[row] < 16) T.add((uint32_t)row / 16, (uint32_t)row % 16, 0, 0);
    for (int i = 0; i < 4096; i++) tab[i] = (uint8_t)(T.e[i] & 0xff);
}

// Time factors of tiled geometries: eight GPU melts of N=100 rings (density
// 1.2) against the eight reference efpol melts at L=64, the centre-of-mass
// MSD over steps 15000-50000 at lags of 500 to 25000 steps; f is the step
// ratio that maps the GPU's MSD curve onto efpol's (log-log interpolation),
// the same at every lag within its error of 0.001-0.005
// (tests/test_gpu_stats.py checks three shapes).  The GPU melts run at L=64
// where the shape divides it, else at L=48 (48x24x24, 24^3) or L=80
// (40x20x20, 20^3): efpol runs powers of two only, and ring motion at N=100
// does not depend on the box at these sizes.  Equilibrium statistics of all
// these runs agree with efpol's within their errors.  Every shape the
// default geometry can take is listed.
namespace {
struct TimeFactor {
    int tx, ty, tz;
    double f;
};
const TimeFactor kTimeFactors[] = {
    {32, 32, 32, 0.926},
    {48, 24, 24, 0.914},
    {32, 32, 16, 0.899},
    {24, 24, 24, 0.900},
    {40, 20, 20, 0.900},
    {20, 20, 20, 0.884},
    {32, 16, 16, 0.877},
    {16, 16, 16, 0.855},
    {16, 16, 8, 0.800},
};
}  // namespace

extern "C" double elp_time_factor(int32_t periodic, int32_t tx, int32_t ty, int32_t tz)
{
    if (periodic) return 1.0;
    for (const TimeFactor& t : kTimeFactors)
        if (t.tx == tx && t.ty == ty && t.tz == tz) return t.f;
    return 0.0;
}

// GetNPol, cpupol/efpol_lib.c:50-56
int elp_get_npol(double density, int N, long sites)
{
    return (int)(density * (double)sites / (double)N + 0.5);
}

// CreatePolymers, cpupol/efpol_init.c:239-283: chains on a delta-spaced
// grid (monomer 0 alone, bond +v, the other N-1 monomers stored on the next
// site; the site words are written by init_kernel, elp_build.cu).  The
// grid's spacing and extents; returns 0, or 1 if it cannot hold P chains.
int elp_initial_grid(int L, int N, int P, int* delta_out, int* nt_out, int* nv_out)
{
    if (N < 3 || P < 1) return 1;
    int delta;
    for (delta = 1; delta < L; delta++) {
        long ntot = (long)(L / delta) * (L / delta) * (L / (delta + 1));
        if (ntot < P) { delta--; break; }
    }
    // every spacing fits (a handful of chains): the reference's loop runs out
    // here and divides by zero; take the widest spacing, L - 1
    if (delta >= L) delta = L - 1;
    if (delta < 1) return 1;
    int nt = L / delta, nv = L / (delta + 1);
    if ((long)nt * nv * (L / delta) < P) return 1;
    *delta_out = delta;
    *nt_out = nt;
    *nv_out = nv;
    return 0;
}

