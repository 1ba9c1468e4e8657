// elp_double.cpp -- hierarchical doubling of a ring melt (host code).
//
// efpol builds large melts by equilibrating a small one and doubling it
// (DoubleLattice, cpupol/efpol_init.c:114-207, driven by cpupol/efpol.c:90-101):
// the box edge doubles and every monomer becomes eight, so ring length grows
// 8x at the same density.  A monomer at r whose bond to the next monomer is
// u becomes four monomers at 2r, a bond u, four monomers at 2r + u and a bond
// u, which ends at 2(r + u), the image of the next monomer.
//
// A ring that occupies exactly two sites (two non-zero bonds u and -u, the
// compact state every ring starts in) would double into a ring that retraces
// itself; it is rebuilt instead as five runs with bonds u, u, d1, -u, d3
// from 2r0, r0 the site of the first monomer whose bond u has no w
// component.  (d1, d3) is option `try` = 0..3 of the transition table's row
// (0, -u), the first whose two new sites are free among everything doubled
// so far (rings in index order); the 8N monomers are spread over the five
// runs as N8/5 each plus one for the first N8 % 5 runs.  Monomer 0 of the
// rebuilt ring sits at 2r0.
#include <stdio.h>
#include <string.h>

#include <vector>

#include "elp_common.h"

namespace {

struct Box {
    int L;
    int t, u, v;
    void step(uint32_t b)
    {
        t += elp_bt(b); u += elp_bu(b); v += elp_bv(b);
        t = (t % L + L) % L; u = (u % L + L) % L; v = (v % L + L) % L;
    }
    size_t index() const { return (size_t)t + (size_t)L * ((size_t)u + (size_t)L * (size_t)v); }
};

}  // namespace

extern "C" elp_status elp_double_chains(int32_t L, int32_t N, int32_t P, const int32_t* start, const uint8_t* bonds,
                                        int32_t* start_out, uint8_t* bonds_out)
{
    if (!start || !bonds || !start_out || !bonds_out) return elp_fail(ELP_ERR_ARG, "null argument");
    if (L < 2 || L > 512 || N < 1 || P < 1 || (long long)N * 8 > ELP_MAX_N)
        return elp_fail(ELP_ERR_ARG, "cannot double L=%d N=%d P=%d (8N must be at most %d)", L, N, P, ELP_MAX_N);
    const int L2 = 2 * L;
    const int N8 = 8 * N;
    uint8_t table[4096];
    elp_status st = elp_transition_table(table);
    if (st) return st;
    std::vector<uint8_t> occ;
    try {
        occ.assign((size_t)L2 * L2 * L2, 0);
    } catch (...) {
        return elp_fail(ELP_ERR_NOMEM, "out of host memory");
    }
    for (int p = 0; p < P; p++) {
        const uint8_t* b = bonds + (size_t)p * N;
        uint8_t* bo = bonds_out + (size_t)p * N8;
        const int32_t* s = start + 3 * (size_t)p;
        for (int m = 0; m < N; m++) {
            if (b[m] > 15) return elp_fail(ELP_ERR_ARG, "ring %d: bond code %d is not 4-bit", p, b[m]);
            if (b[m] == 15) return elp_fail(ELP_ERR_ARG, "chain %d ends in 0xf: DoubleLattice doubles rings only", p);
        }
        if (s[0] < 0 || s[0] >= L || s[1] < 0 || s[1] >= L || s[2] < 0 || s[2] >= L)
            return elp_fail(ELP_ERR_ARG, "ring %d: start outside the box", p);
        // the plain doubling, which also marks the doubled sites occupied
        Box r{L, s[0], s[1], s[2]};
        int nunit = 0;
        memset(bo, 0, (size_t)N8);
        for (int m = 0; m < N; m++) {
            const uint32_t u = b[m];
            nunit += u ? 1 : 0;
            Box d{L2, 2 * r.t, 2 * r.u, 2 * r.v};
            occ[d.index()] = 1;
            bo[8 * m + 3] = (uint8_t)u;
            bo[8 * m + 7] = (uint8_t)u;
            d.step(u);
            occ[d.index()] = 1;
            r.step(u);
        }
        start_out[3 * (size_t)p + 0] = 2 * s[0];
        start_out[3 * (size_t)p + 1] = 2 * s[1];
        start_out[3 * (size_t)p + 2] = 2 * s[2];
        if (nunit != 2) continue;

        // a two-site ring: rebuild it as five runs around 2 r0
        Box r0{L, s[0], s[1], s[2]};
        uint32_t unit = 0;
        for (int m = 0; m < N; m++) {
            if (b[m] && b[m] < 8) {
                unit = b[m];
                break;
            }
            r0.step(b[m]);
        }
        const uint32_t combo = (~unit) & 15u;
        bool placed = false;
        for (int attempt = 0; attempt < 4 && !placed; attempt++) {
            const uint8_t e = table[(combo << 4) | (uint32_t)attempt];
            const uint32_t units[5] = {unit, unit, (uint32_t)(e & 15), combo, (uint32_t)(e >> 4)};
            Box c{L2, 2 * r0.t, 2 * r0.u, 2 * r0.v};
            size_t saved[5] = {0, 0, 0, 0, 0};
            int mono = 0;
            bool clash = false;
            for (int i = 0; i < 5 && !clash; i++) {
                const int cnt = N8 / 5 + (i < N8 % 5 ? 1 : 0);
                for (int j = 0; j + 1 < cnt; j++) bo[mono++] = 0;
                bo[mono++] = (uint8_t)units[i];
                c.step(units[i]);
                if (i >= 2 && i < 4 && occ[c.index()]) {
                    for (int k = 2; k < i; k++) occ[saved[k]] = 0;
                    clash = true;
                    break;
                }
                occ[c.index()] = 1;
                saved[i] = c.index();
                if (i == 4) placed = true;
            }
        }
        if (!placed)
            return elp_fail(ELP_ERR_STATE, "ring %d: no free sites to rebuild its two-site doubling", p);
        start_out[3 * (size_t)p + 0] = 2 * r0.t;
        start_out[3 * (size_t)p + 1] = 2 * r0.u;
        start_out[3 * (size_t)p + 2] = 2 * r0.v;
    }
    return ELP_OK;
}
