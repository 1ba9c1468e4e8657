// elp_scaleup.cpp -- upscaling of a ring melt's TUV file to a box of twice
// the edge and rings of eight times the length: the doubling step of the
// reference's GPU runs (do_run.sh:290-330 calls analysis/scaleup.c).
//
// Every occupied site of the coarse ring becomes a 2x2x2 cube of fine sites
// walked by a self-avoiding path of seven bonds; consecutive cubes are joined
// by one fine bond between an exit corner of one cube and an entry corner
// of the next, so the coarse bond from cube A to cube B fixes which corner
// pairs can be joined ("ports").  The steps, which must match the reference
// to give the same file, are:
//   1. enumerate, for every (entry, exit) corner pair, all seven-bond paths
//      through the cube's eight corners, depth first with bond codes tried in
//      ascending order (analysis/scaleup.c:103-146);
//   2. for every coarse bond, list the (exit corner, entry corner, fine bond)
//      triples that realise it (scaleup.c:44-86);
//   3. per ring, with one Tausworthe stream (util/rng.h:10-35) seeded with
//      192869123 for the whole file: assign ports by priority -- a bond whose
//      candidate triples leave fewer distinct choices is fixed first, each
//      examination drawing one random number (scaleup.c:150-205); then pick
//      one enumerated path per cube at random (scaleup.c:250-268);
//   4. zero bonds (stored length) of the coarse ring are repeated after every
//      fine monomer of the cube that holds them; the ring starts at the entry
//      corner of the first cube.
// Output: the TUV header with 2L and 8 * maxPolLength, then per ring
// "len= <n>", "t u v" and the bond string on three lines.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <array>
#include <string>
#include <vector>

#include "elp_common.h"
#include "elp_taus.h"

namespace {

using Taus = elp_taus;

using Path = std::array<uint8_t, 7>;

struct CubePaths {
    std::vector<Path> by_pair[64];   // index entry + 8 * exit
};

void cube_walk(CubePaths& cp, int used, int pos, int entry, int depth, Path& path)
{
    if (used & (1 << pos)) return;
    if (depth == 7) {
        cp.by_pair[entry + 8 * pos].push_back(path);
        return;
    }
    used |= 1 << pos;
    for (uint32_t b = 1; b < 15; b++) {
        if (!elp_valid_bond(b)) continue;
        int np;
        if (b & 8) {   // components -1 on the bits b lacks: those corners bits must be set
            if ((~(b | (uint32_t)pos)) & 7u) continue;
            np = (int)(((uint32_t)pos ^ ~b) & 7u);
        } else {       // components +1 on b's bits: those corner bits must be clear
            if (b & (uint32_t)pos) continue;
            np = pos | (int)b;
        }
        path[(size_t)depth] = (uint8_t)b;
        cube_walk(cp, used, np, entry, depth + 1, path);
    }
}

struct PortTriple {
    int exit, entry, bond;
};

// Cube paths and port triples, built once (thread-safe static initialisation).
struct Tables {
    CubePaths cp;
    std::vector<PortTriple> port_triples[16];
    Tables();
};

const Tables& tables()
{
    static const Tables t;
    return t;
}

Tables::Tables()
{
    Path path{};
    for (int e = 0; e < 8; e++) cube_walk(cp, 0, e, e, 0, path);
    for (uint32_t b = 1; b < 15; b++) {
        if (!elp_valid_bond(b)) continue;
        const int dt = elp_bt(b), du = elp_bu(b), dv = elp_bv(b);
        for (int pos = 0; pos < 8; pos++) {
            const int tp = pos & 1, up = (pos >> 1) & 1, vp = (pos >> 2) & 1;
            for (uint32_t nb = 1; nb < 15; nb++) {
                if (!elp_valid_bond(nb)) continue;
                const int nt = tp + elp_bt(nb), nu = up + elp_bu(nb), nv = vp + elp_bv(nb);
                // fine coordinate -1..2 lies in cube floor(c / 2) of the coarse step
                if ((nt + 2) / 2 - 1 != dt || (nu + 2) / 2 - 1 != du || (nv + 2) / 2 - 1 != dv) continue;
                const int npos = ((nt + 2) % 2) + 2 * ((nu + 2) % 2) + 4 * ((nv + 2) % 2);
                port_triples[b].push_back(PortTriple{pos, npos, (int)nb});
            }
        }
    }
}

// One random triple for a coarse bond whose neighbours already use the
// given corners; returns its priority (1 + fewest distinct exit or entry
// corners among the candidates, 1 if only one), 0 if none is possible.
int random_triple(int bond, int used_exit_neighbour, int used_entry_neighbour, Taus& rng, PortTriple* out)
{
    PortTriple cand[16];
    int n = 0;
    for (const PortTriple& t : tables().port_triples[bond]) {
        if (t.exit == used_exit_neighbour || t.entry == used_entry_neighbour) continue;
        if (n < 16) cand[n] = t;
        n++;
    }
    if (n == 0 || n > 16) return 0;
    int ndif_exit = 1, ndif_entry = 1;
    for (int i = 1; i < n; i++) {
        if (cand[i].exit != cand[0].exit) ndif_exit++;
        if (cand[i].entry != cand[0].entry) ndif_entry++;
    }
    *out = cand[rng.below(n)];
    if (n == 1) return 1;
    return 1 + (ndif_exit < ndif_entry ? ndif_exit : ndif_entry);
}

bool next_token(const char*& p, std::string& tok)
{
    while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') p++;
    if (!*p) return false;
    const char* b = p;
    while (*p && *p != ' ' && *p != '\t' && *p != '\n' && *p != '\r') p++;
    tok.assign(b, (size_t)(p - b));
    return true;
}

bool next_int(const char*& p, long* v)
{
    std::string t;
    if (!next_token(p, t)) return false;
    char* e = nullptr;
    *v = strtol(t.c_str(), &e, 10);
    return e && *e == '\0';
}

}  // namespace

extern "C" elp_status elp_scaleup_tuv(const char* in_path, const char* out_path)
{
    if (!in_path || !out_path) return elp_fail(ELP_ERR_ARG, "null argument");
    char* text = nullptr;
    size_t tlen = 0;
    elp_status st = elp_read_file(in_path, &text, &tlen);
    if (st) return st;
    std::string out;
    const CubePaths& cp = tables().cp;
    Taus rng(192869123u);
    const char* p = text;
    std::string tok;
    long lt, lu, lv, np, maxlen;
    bool ok = next_token(p, tok) && next_int(p, &lt) && next_token(p, tok) && next_int(p, &lu) &&
              next_token(p, tok) && next_int(p, &lv) && next_token(p, tok) && next_int(p, &np) &&
              next_token(p, tok) && next_int(p, &maxlen);
    if (!ok || np < 1 || maxlen < 1) {
        free(text);
        return elp_fail(ELP_ERR_FORMAT, "%s: not a TUV file", in_path);
    }
    char line[128];
    snprintf(line, sizeof(line), "LT= %ld\nLU= %ld\nLV= %ld\nnp= %ld\nmaxPolLength= %ld\n", 2 * lt, 2 * lu, 2 * lv,
             np, 8 * maxlen);
    out += line;
    std::vector<int> bonds, nsl, ports;
    std::vector<char> fine;
    static const char hexd[] = "0123456789abcdef";
    for (long ip = 0; ip < np; ip++) {
        long len, t, u, v;
        if (!(next_token(p, tok) && next_int(p, &len) && next_int(p, &t) && next_int(p, &u) && next_int(p, &v) &&
              next_token(p, tok)) || len < 1 || (long)tok.size() != len) {
            free(text);
            return elp_fail(ELP_ERR_FORMAT, "%s: ring %ld is malformed", in_path, ip);
        }
        // coarse non-zero bonds; nsl[i] zero bonds (stored monomers) before bond i,
        // the trailing ones belong to the first site
        bonds.clear();
        nsl.assign((size_t)len + 1, 0);
        for (long i = 0; i < len; i++) {
            const char c = tok[(size_t)i];
            const int b = (c >= '0' && c <= '9') ? c - '0' : ((c >= 'a' && c <= 'f') ? 10 + c - 'a' : -1);
            if (b < 0 || (b && !elp_valid_bond((uint32_t)b))) {
                free(text);
                return elp_fail(ELP_ERR_FORMAT, "%s: ring %ld has bond '%c'", in_path, ip, c);
            }
            if (!b) nsl[bonds.size()]++;
            else bonds.push_back(b);
        }
        const int nb = (int)bonds.size();
        if (nb < 2) {
            free(text);
            return elp_fail(ELP_ERR_FORMAT, "%s: ring %ld has fewer than two sites", in_path, ip);
        }
        nsl[0] += nsl[(size_t)nb];
        // ports: exit corner (2i) and entry corner (2i+1) of coarse bond i
        ports.assign((size_t)2 * nb, -1);
        for (;;) {
            int nset = 0;
            for (int prio = 1, nprio = 0; prio < 10 && !nprio; prio++) {
                for (int i = 0; i < nb; i++) {
                    if (ports[(size_t)2 * i] >= 0) continue;
                    const int used_exit = ports[(size_t)((2 * i - 1 + 2 * nb) % (2 * nb))];
                    const int used_entry = ports[(size_t)((2 * i + 2) % (2 * nb))];
                    PortTriple tr{};
                    const int cur = random_triple(bonds[(size_t)i], used_exit, used_entry, rng, &tr);
                    if (cur == 0) {
                        free(text);
                        return elp_fail(ELP_ERR_STATE, "%s: ring %ld: no corner pair for bond %d", in_path, ip, i);
                    }
                    if (cur == prio) {
                        ports[(size_t)2 * i] = tr.exit;
                        ports[(size_t)2 * i + 1] = tr.entry;
                        bonds[(size_t)i] = tr.bond;
                        nset++;
                        nprio++;
                    }
                }
            }
            if (!nset) break;
        }
        for (int i = 0; i < 2 * nb; i++)
            if (ports[(size_t)i] < 0) {
                free(text);
                return elp_fail(ELP_ERR_STATE, "%s: ring %ld: corners left unassigned", in_path, ip);
            }
        fine.clear();
        for (int i = 0; i < nb; i++) {
            const int entry = ports[(size_t)((2 * i - 1 + 2 * nb) % (2 * nb))];
            const int exit = ports[(size_t)2 * i];
            const std::vector<Path>& paths = cp.by_pair[entry + 8 * exit];
            if (paths.empty()) {
                free(text);
                return elp_fail(ELP_ERR_STATE, "%s: ring %ld: no cube path %d -> %d", in_path, ip, entry, exit);
            }
            const Path& path = paths[(size_t)rng.below((int)paths.size())];
            for (int k = 0; k < 7; k++) {
                fine.push_back(hexd[path[(size_t)k]]);
                fine.insert(fine.end(), (size_t)nsl[(size_t)i], '0');
            }
            fine.push_back(hexd[bonds[(size_t)i]]);
            fine.insert(fine.end(), (size_t)nsl[(size_t)i], '0');
        }
        const int e0 = ports[(size_t)2 * nb - 1];
        snprintf(line, sizeof(line), "len= %zu\n%ld %ld %ld\n", fine.size(), 2 * t + (e0 & 1), 2 * u + ((e0 >> 1) & 1),
                 2 * v + ((e0 >> 2) & 1));
        out += line;
        out.append(fine.data(), fine.size());
        out += '\n';
    }
    free(text);
    FILE* f = fopen(out_path, "wb");
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", out_path);
    const bool wr = fwrite(out.data(), 1, out.size(), f) == out.size();
    if (fclose(f) || !wr) return elp_fail(ELP_ERR_IO, "short write to %s", out_path);
    return ELP_OK;
}
