// elp_pov.cpp -- export of a TUV file as a POV-Ray scene, the visualisation
// feed of the reference's analysis/tuv2pov.c (rendered by an external
// POV-Ray; this writes the scene text only).  The output is the reference's
// byte for byte:
//
//   * chains are walked from their start site along their bonds; a monomer
//     stored on its predecessor's site adds no position (tuv2pov.c:162-172);
//     positions are x = (t+u-v)/sqrt 2, y = (t-u)/sqrt 2, z = v/sqrt 2;
//   * the camera looks at the mean position of the drawn chains along the
//     fixed direction (0.72347, 0.502397, 0.224491), far enough back that a
//     15 degree view holds every monomer, by the reference's own distance
//     rule (tuv2pov.c:351-398); the area light sits at the same distance,
//     40 degrees off the view axis about an orthogonal axis drawn from the
//     reference's fixed Tausworthe stream (seed 1029471, tuv2pov.c:292-328);
//   * per chain a merge of cylinders between consecutive positions and a
//     sphere at every site not drawn before (any chain), coloured by chain
//     (all chains) or along the chain (one chain), tuv2pov.c:204-233.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <unordered_set>
#include <vector>

#include "elp_common.h"
#include "elp_taus.h"

namespace {

// the reference's value of pi (analysis/lowm_modes.h:16)
constexpr double kPi = 3.14159265359;

struct V3 {
    double x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scale(double s, V3 c) { return {c.x * s, c.y * s, c.z * s}; }
V3 axpy(double a, V3 v1, V3 v2) { return {a * v1.x + v2.x, a * v1.y + v2.y, a * v1.z + v2.z}; }
double dot(V3 a, V3 b)
{
    double r = 0;
    r += a.x * b.x;
    r += a.y * b.y;
    r += a.z * b.z;
    return r;
}
V3 unit(V3 c)
{
    const double n = sqrt(dot(c, c));
    return {c.x / n, c.y / n, c.z / n};
}

// A random unit vector at least 60 degrees off `u` (and off `w` when given),
// made orthogonal to them; every call restarts the same stream.
V3 random_orthogonal(V3 u)
{
    elp_taus rng(1029471u);
    V3 c;
    do {
        c.x = 2 * rng.uniform() - 1;
        c.y = 2 * rng.uniform() - 1;
        c.z = 2 * rng.uniform() - 1;
        c = unit(c);
    } while (fabs(dot(c, u)) > 0.5);
    c = axpy(-dot(c, u), u, c);
    return unit(c);
}
void two_orthogonal(V3 u, V3* o1, V3* o2)
{
    *o1 = random_orthogonal(u);
    elp_taus rng(1029471u);
    V3 c;
    do {
        c.x = 2 * rng.uniform() - 1;
        c.y = 2 * rng.uniform() - 1;
        c.z = 2 * rng.uniform() - 1;
        c = unit(c);
    } while (fabs(dot(c, u)) > 0.5 || fabs(dot(c, *o1)) > 0.5);
    c = axpy(-dot(c, u), u, c);
    *o2 = unit(axpy(-dot(c, *o1), *o1, c));
}

// Rotation of v by `deg` degrees about the unit axis a (Rodrigues' matrix,
// accumulated row by row).
V3 rotate(V3 a, double deg, V3 v)
{
    const double ang = deg * 2 * kPi / 360;
    const double c = cos(ang), s = sin(ang), C = 1 - c;
    V3 r = {0, 0, 0};
    r.x += v.x * (a.x * a.x * C + c);
    r.x += v.y * (a.x * a.y * C - a.z * s);
    r.x += v.z * (a.x * a.z * C + a.y * s);
    r.y += v.x * (a.y * a.x * C + a.z * s);
    r.y += v.y * (a.y * a.y * C + c);
    r.y += v.z * (a.y * a.z * C - a.x * s);
    r.z += v.x * (a.z * a.x * C - a.y * s);
    r.z += v.y * (a.z * a.y * C + a.x * s);
    r.z += v.z * (a.z * a.z * C + c);
    return r;
}

// Colour ramp of the reference: 0 -> 1 -> 1 -> 0 over quarters of a period.
double ramp(double f)
{
    f -= (int)f;
    if (f < 0.25) return 4 * f;
    if (f < 0.5) return 1;
    if (f < 0.75) return 3 - 4 * f;
    return 0;
}

struct Chain {
    std::vector<int> tuv;   // 3 per position
    std::vector<V3> pos;
};

void write_pos(FILE* f, V3 c) { fprintf(f, " <%lf, %lf, %lf> ", c.x, c.y, c.z); }

}  // namespace

extern "C" elp_status elp_tuv_to_pov(const char* in_path, const char* out_path, int32_t pol_id)
{
    if (!in_path || !out_path) return elp_fail(ELP_ERR_ARG, "null argument");
    char* text = nullptr;
    size_t len = 0;
    elp_status st = elp_read_file(in_path, &text, &len);
    if (st) return st;
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
    for (int i = 0; i < 8; i++)
        if (!token(tok)) return elp_fail(ELP_ERR_FORMAT, "%s: not a TUV file", in_path);
    const long npol = strtol(tok.c_str(), nullptr, 10);
    if (!token(tok) || !token(tok)) return elp_fail(ELP_ERR_FORMAT, "%s: not a TUV file", in_path);
    if (npol < 1) return elp_fail(ELP_ERR_FORMAT, "%s: np= %ld", in_path, npol);
    if (pol_id >= npol) return elp_fail(ELP_ERR_ARG, "chain %d does not exist (np= %ld)", pol_id, npol);
    const bool all = pol_id < 0;

    std::vector<Chain> ch((size_t)npol);
    for (long c = 0; c < npol; c++) {
        std::string lenword, n, t, u, v, bonds;
        if (!token(lenword) || !token(n) || !token(t) || !token(u) || !token(v) || !token(bonds))
            return elp_fail(ELP_ERR_FORMAT, "%s: chain %ld truncated", in_path, c);
        const long nmono = strtol(n.c_str(), nullptr, 10);
        if (nmono < 1 || (size_t)nmono > bonds.size())
            return elp_fail(ELP_ERR_FORMAT, "%s: chain %ld has len= %ld", in_path, c, nmono);
        int x[3] = {(int)strtol(t.c_str(), nullptr, 10), (int)strtol(u.c_str(), nullptr, 10),
                    (int)strtol(v.c_str(), nullptr, 10)};
        Chain& k = ch[(size_t)c];
        for (long i = 0; i < nmono; i++) {
            const char bc = bonds[(size_t)i];
            const uint32_t b = (uint32_t)((bc >= '0' && bc <= '9') ? bc - '0' : 10 + bc - 'a') & 15u;
            if (!(i && bonds[(size_t)i - 1] == '0')) {
                k.tuv.insert(k.tuv.end(), x, x + 3);
                k.pos.push_back({(x[0] + x[1] - x[2]) / sqrt(2.0), (x[0] - x[1]) / sqrt(2.0), x[2] / sqrt(2.0)});
            }
            x[0] += elp_bt(b); x[1] += elp_bu(b); x[2] += elp_bv(b);
        }
    }

    // camera
    const V3 view = unit({0.72347, 0.502397, 0.224491});
    V3 look = {0, 0, 0};
    long navg = 0;
    for (long c = 0; c < npol; c++) {
        if (!all && c != pol_id) continue;
        for (const V3& q : ch[(size_t)c].pos) { look = add(look, q); navg++; }
    }
    look.x /= navg; look.y /= navg; look.z /= navg;
    double angle = 15;
    const double cosfac = tan((angle / 2.0 - 0.5) / 360.0 * 2 * kPi);
    double maxd = 0.0;
    for (long c = 0; c < npol; c++) {
        if (!all && c != pol_id) continue;
        for (const V3& q : ch[(size_t)c].pos) {
            const V3 z = sub(q, look);
            double dx = dot(z, view);
            dx = dx < 0 ? -sqrt(-dx) : sqrt(dx);
            const V3 yv = sub(z, scale(dx, view));
            const double x = sqrt(dot(yv, yv)) / cosfac;
            if (x + dx > maxd) maxd = x + dx;
        }
    }
    const V3 cam = axpy(maxd, view, look);
    angle += 0.5;
    const V3 light_dir = rotate(random_orthogonal(view), 40, view);
    const V3 light = axpy(maxd, light_dir, look);
    V3 o1, o2;
    two_orthogonal(light_dir, &o1, &o2);
    const V3 area1 = scale(0.1 * maxd, o1), area2 = scale(0.1 * maxd, o2);

    FILE* f = fopen(out_path, "w");
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", out_path);
    fprintf(f, "light_source { <%lf, %lf, %lf> ", light.x, light.y, light.z);
    fprintf(f, "color White area_light <%lf,%lf,%lf>,", area1.x, area1.y, area1.z);
    fprintf(f, "<%lf,%lf,%lf>, 3, 3\n\tadaptive 5\n}\n", area2.x, area2.y, area2.z);
    fprintf(f, "camera { location ");
    write_pos(f, cam);
    fprintf(f, "up y\n right x\n");
    fprintf(f, "angle %lf \n", angle);
    fprintf(f, "look_at ");
    write_pos(f, look);
    fprintf(f, "}\n");

    const double size = 0.15;
    std::unordered_set<uint64_t> drawn;   // sites with a sphere (unwrapped coordinates)
    auto site_key = [](const int* x) {
        return ((uint64_t)(uint32_t)(x[0] + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(x[1] + (1 << 20)) << 21) |
               (uint64_t)(uint32_t)(x[2] + (1 << 20));
    };
    char color[128] = "";
    bool ok = true;
    for (long c = 0; c < npol && ok; c++) {
        if (!all && c != pol_id) continue;
        const Chain& k = ch[(size_t)c];
        const long n = (long)k.pos.size();
        fprintf(f, "\nmerge {\n");
        for (long i = 0; i < n; i++) {
            if (i < n - 1) {
                double rgb[3];
                if (!all) {
                    const double fr = i / (double)n;
                    rgb[0] = ramp(fr); rgb[1] = ramp(fr + 0.25); rgb[2] = ramp(fr + 0.5);
                } else {
                    const double fc = c / (double)npol, white = 0.3 * (i / (double)n);
                    rgb[0] = ramp(fc); rgb[1] = ramp(fc + 0.25); rgb[2] = ramp(fc + 0.5);
                    for (int q = 0; q < 3; q++) rgb[q] = white + (1 - white) * rgb[q];
                }
                snprintf(color, sizeof(color), "rgbf<%lf, %lf, %lf>", rgb[0], rgb[1], rgb[2]);
            }
            // the last position keeps the colour of the last link
            if (drawn.insert(site_key(&k.tuv[3 * (size_t)i])).second) {
                fprintf(f, "object { sphere { ");
                write_pos(f, k.pos[(size_t)i]);
                fprintf(f, ", %lf texture {pigment {color %s}} finish {ambient 0.1 diffuse 0.6} } }\n", 1.5 * size,
                        color);
            }
            if (i < n - 1) {
                fprintf(f, "object { cylinder {");
                write_pos(f, k.pos[(size_t)i]);
                fprintf(f, ", ");
                write_pos(f, k.pos[(size_t)i + 1]);
                ok = fprintf(f, ", %lf texture {pigment {color %s}} finish { ambient 0.1 diffuse 0.6} } } \n", size,
                             color) > 0;
            }
        }
        fprintf(f, "}\n");
    }
    if (fclose(f) || !ok) return elp_fail(ELP_ERR_IO, "short write to %s", out_path);
    return ELP_OK;
}
