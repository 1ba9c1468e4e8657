// elp_ptl.cpp -- per-ring time series ("PTL" files) written during a run.
//
// The reference's analysis first transposes a run's TUV dumps into one file
// per ring, sample_dir/ptl/pol=<p>_dev=<d>.res (analysis/create_ptl.c:46-115):
//
//     polId= <p>
//     nTime= <number of dumps>
//     len= <N>
//     <t> <u> <v> <bond hex string>        one line per dump, oldest first
//
// and its mode analysis reads those (LoadPTL, analysis/mode_io.c:509-606).
// This writer produces the same files while the run dumps, so the
// transposition pass has nothing left to do.  Lines are kept in host memory
// and appended to the files when the buffer fills and at close, which keeps
// the number of open files at one.
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <new>
#include <string>
#include <vector>

#include "elp_common.h"

struct elp_ptl {
    std::string dir;                  // sample_dir/ptl
    int dev = 0, P = 0, N = 0, ntime = 0;
    int appended = 0;                 // dumps appended so far
    size_t budget = 0, held = 0;      // buffered bytes
    std::vector<std::string> lines;   // pending text per ring
    std::vector<char> started;        // file created (header written) per ring
};

static int mkdir_p(const std::string& path)
{
    std::string cur;
    for (size_t i = 0; i <= path.size(); i++) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) && errno != EEXIST) return -1;
        }
        if (i < path.size()) cur.push_back(path[i]);
    }
    return 0;
}

static elp_status ptl_flush(elp_ptl* w)
{
    char name[64];
    for (int p = 0; p < w->P; p++) {
        std::string& s = w->lines[(size_t)p];
        if (s.empty() && w->started[(size_t)p]) continue;
        snprintf(name, sizeof(name), "/pol=%d_dev=%d.res", p, w->dev);
        const std::string path = w->dir + name;
        FILE* f = fopen(path.c_str(), w->started[(size_t)p] ? "ab" : "wb");
        if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", path.c_str());
        bool ok = true;
        if (!w->started[(size_t)p]) ok = fprintf(f, "polId= %d\nnTime= %d\nlen= %d\n", p, w->ntime, w->N) > 0;
        if (ok && !s.empty()) ok = fwrite(s.data(), 1, s.size(), f) == s.size();
        if (fclose(f) || !ok) return elp_fail(ELP_ERR_IO, "short write to %s", path.c_str());
        w->started[(size_t)p] = 1;
        std::string().swap(s);
    }
    w->held = 0;
    return ELP_OK;
}

extern "C" elp_status elp_ptl_open(const char* sample_dir, int32_t dev, int32_t P, int32_t N, int32_t ntime,
                                   size_t buffer_bytes, elp_ptl** out)
{
    if (!sample_dir || !out) return elp_fail(ELP_ERR_ARG, "null argument");
    *out = nullptr;
    if (dev < 0 || P < 1 || N < 1 || ntime < 1)
        return elp_fail(ELP_ERR_ARG, "bad PTL shape dev=%d P=%d N=%d ntime=%d", dev, P, N, ntime);
    elp_ptl* w = new (std::nothrow) elp_ptl();
    if (!w) return elp_fail(ELP_ERR_NOMEM, "out of host memory");
    w->dir = std::string(sample_dir) + "/ptl";
    w->dev = dev; w->P = P; w->N = N; w->ntime = ntime;
    w->budget = buffer_bytes ? buffer_bytes : ((size_t)256 << 20);
    try {
        w->lines.resize((size_t)P);
        w->started.assign((size_t)P, 0);
    } catch (...) {
        delete w;
        return elp_fail(ELP_ERR_NOMEM, "out of host memory");
    }
    if (mkdir_p(w->dir)) {
        elp_status st = elp_fail(ELP_ERR_IO, "cannot create %s", w->dir.c_str());
        delete w;
        return st;
    }
    *out = w;
    return ELP_OK;
}

extern "C" elp_status elp_ptl_append(elp_ptl* w, const int32_t* start, const uint8_t* bonds)
{
    if (!w || !start || !bonds) return elp_fail(ELP_ERR_ARG, "null argument");
    if (w->appended >= w->ntime)
        return elp_fail(ELP_ERR_STATE, "all %d dumps of the PTL files are written", w->ntime);
    static const char hexd[] = "0123456789abcdef";
    char head[48];
    for (int p = 0; p < w->P; p++) {
        const uint8_t* b = bonds + (size_t)p * w->N;
        for (int i = 0; i < w->N; i++)
            if (b[i] > 15) return elp_fail(ELP_ERR_ARG, "ring %d: bond code %d is not 4-bit", p, b[i]);
    }
    try {
        for (int p = 0; p < w->P; p++) {
            std::string& s = w->lines[(size_t)p];
            int n = snprintf(head, sizeof(head), "%d %d %d ", start[3 * (size_t)p], start[3 * (size_t)p + 1],
                             start[3 * (size_t)p + 2]);
            const size_t before = s.size();
            s.append(head, (size_t)n);
            const uint8_t* b = bonds + (size_t)p * w->N;
            for (int i = 0; i < w->N; i++) s.push_back(hexd[b[i]]);
            s.push_back('\n');
            w->held += s.size() - before;
        }
    } catch (...) {
        return elp_fail(ELP_ERR_NOMEM, "out of host memory");
    }
    w->appended++;
    if (w->held >= w->budget) return ptl_flush(w);
    return ELP_OK;
}

extern "C" elp_status elp_ptl_close(elp_ptl* w)
{
    if (!w) return ELP_OK;
    elp_status st = ptl_flush(w);
    const int appended = w->appended, ntime = w->ntime;
    delete w;
    if (st) return st;
    if (appended != ntime)
        return elp_fail(ELP_ERR_STATE, "PTL files announce %d dumps but %d were appended", ntime, appended);
    return ELP_OK;
}
