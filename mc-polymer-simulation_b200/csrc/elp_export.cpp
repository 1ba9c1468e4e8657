// elp_export.cpp -- export of one ring of a TUV file as xyz coordinates, the
// visualisation feed of the reference's analysis/tuv2xyz.c: one line
// "x y z" per monomer ("%lf" each), x = (t+u-v)/sqrt(2), y = (t-u)/sqrt(2),
// z = v/sqrt(2), positions walked from (0,0,0) along the ring's bonds.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "elp_common.h"

extern "C" elp_status elp_tuv_to_xyz(const char* in_path, int32_t pol_id, const char* out_path)
{
    if (!in_path || !out_path) return elp_fail(ELP_ERR_ARG, "null argument");
    char* text = nullptr;
    size_t len = 0;
    elp_status st = elp_read_file(in_path, &text, &len);
    if (st) return st;
    // header: LT= L LU= L LV= L np= P maxPolLength= N, then per ring "len= n t u v bonds"
    std::string s(text, len);
    free(text);
    const char* p = s.c_str();
    auto token = [&p](std::string& tok) {
        while (*p && strchr(" \t\r\n", *p)) p++;
        const char* b = p;
        while (*p && !strchr(" \t\r\n", *p)) p++;
        tok.assign(b, (size_t)(p - b));
        return !tok.empty();
    };
    std::string tok;
    for (int i = 0; i < 6; i++)
        if (!token(tok)) return elp_fail(ELP_ERR_FORMAT, "%s: not a TUV file", in_path);
    if (!token(tok) || !token(tok)) return elp_fail(ELP_ERR_FORMAT, "%s: not a TUV file", in_path);
    const long npol = strtol(tok.c_str(), nullptr, 10);
    if (pol_id < 0 || pol_id >= npol) return elp_fail(ELP_ERR_ARG, "ring %d does not exist (np= %ld)", pol_id, npol);
    for (int i = 0; i < 2 + 6 * pol_id; i++)
        if (!token(tok)) return elp_fail(ELP_ERR_FORMAT, "%s: truncated", in_path);
    std::string lenword, n, t, u, v, bonds;
    if (!token(lenword) || !token(n) || !token(t) || !token(u) || !token(v) || !token(bonds))
        return elp_fail(ELP_ERR_FORMAT, "%s: ring %d truncated", in_path, pol_id);
    const long nmono = strtol(n.c_str(), nullptr, 10);
    if (nmono < 1 || (size_t)nmono > bonds.size())
        return elp_fail(ELP_ERR_FORMAT, "%s: ring %d has len= %ld", in_path, pol_id, nmono);
    FILE* f = fopen(out_path, "w");
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", out_path);
    long tt = 0, uu = 0, vv = 0;
    bool ok = true;
    for (long i = 0; i < nmono && ok; i++) {
        ok = fprintf(f, "%lf %lf %lf\n", (double)(tt + uu - vv) / sqrt(2.0), (double)(tt - uu) / sqrt(2.0),
                     (double)vv / sqrt(2.0)) > 0;
        const char c = bonds[(size_t)i];
        const uint32_t b = (uint32_t)((c >= '0' && c <= '9') ? c - '0' : 10 + c - 'a') & 15u;
        tt += elp_bt(b); uu += elp_bu(b); vv += elp_bv(b);
    }
    if (fclose(f) || !ok) return elp_fail(ELP_ERR_IO, "short write to %s", out_path);
    return ELP_OK;
}
