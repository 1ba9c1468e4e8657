// elp_common.cu -- see elp_common.h.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "elp_common.h"
#include "elp_kernels.h"

static thread_local std::string g_last_error;

elp_status elp_fail(elp_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

extern "C" const char* elp_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* elp_status_string(elp_status s)
{
    switch (s) {
    case ELP_OK: return "ok";
    case ELP_ERR_ARG: return "invalid argument";
    case ELP_ERR_CUDA: return "CUDA error";
    case ELP_ERR_NOMEM: return "out of memory";
    case ELP_ERR_IO: return "I/O error";
    case ELP_ERR_FORMAT: return "bad TUV format";
    case ELP_ERR_INTEGRITY: return "integrity violation";
    case ELP_ERR_STATE: return "invalid state";
    case ELP_ERR_BUSY: return "busy";
    default: return "unknown status";
    }
}

extern "C" void elp_default_spec(elp_job_spec* s)
{
    memset(s, 0, sizeof(*s));
    s->L = 32;
    s->N = 100;
    s->P = 0;
    s->density = 1.2;
    s->seed = 1;
    s->periodic = -1;
    s->steps_per_launch = 1;
}

// Domain geometry: the whole box on chip when it fits, else a tile shape.
// The first choice depends on the box: attempted moves/s times the shape's
// time factor (the physical rate) was measured for single relaxed melts at
// L = 48, 64, 96, 128, 192, 256, 320 and 512.  Below L = 128, 16^3 tiles
// give the most CTAs and win (L = 64: 13.8 against 12.3 for 32x16x16 and
// 5.5 for 32^3, G moves/s x f); from 128 to 256, 32x16x16 tiles fill the
// SMs at two CTAs each (L = 256: 118 against 111 for 32^3); above 256, the
// 32^3 tiles' slower-wall clock wins (L = 512: 128 against 121).  A box
// that the first choice does not divide takes the first shape of the list
// that does.
static int pick_geometry(const elp_job_spec* s, elp_geometry* g)
{
    const int L = s->L;
    g->L = L;
    if (s->periodic != 0) {
        g->periodic = 1;
        g->tx = g->ty = g->tz = L;
        g->ncol = s->ncol > 0 ? s->ncol : elp_pick_ncol(L);
        if (elp_geometry_ok(g)) return 1;
        if (s->periodic == 1) return 0;
    }
    g->periodic = 0;
    if (s->tile[0] > 0 && s->tile[1] > 0 && s->tile[2] > 0) {
        g->tx = s->tile[0]; g->ty = s->tile[1]; g->tz = s->tile[2];
        g->ncol = s->ncol > 0 ? s->ncol : elp_pick_ncol(g->tx);
        return elp_geometry_ok(g);
    }
    static const int cand[][3] = {{32, 32, 32}, {48, 24, 24}, {32, 32, 16}, {24, 24, 24}, {32, 16, 16},
                                  {16, 16, 16}, {40, 20, 20}, {20, 20, 20}, {16, 16, 8}};
    const int n = (int)(sizeof(cand) / sizeof(cand[0]));
    int order[2 + sizeof(cand) / sizeof(cand[0])];
    int no = 0;
    if (L < 128) order[no++] = 5;                       // 16^3
    else if (L <= 256) { order[no++] = 4; order[no++] = 5; }  // 32x16x16, then 16^3
    for (int i = 0; i < n; i++) order[no++] = i;
    for (int k = 0; k < no; k++) {
        const int i = order[k];
        g->tx = cand[i][0]; g->ty = cand[i][1]; g->tz = cand[i][2];
        if (L % g->tx || L % g->ty || L % g->tz) continue;
        g->ncol = s->ncol > 0 ? s->ncol : elp_pick_ncol(g->tx);
        if (g->ncol && elp_geometry_ok(g)) return 1;
    }
    return 0;
}

elp_status elp_resolve_spec(const elp_job_spec* spec, int* P, elp_geometry* g)
{
    if (!spec) return elp_fail(ELP_ERR_ARG, "null spec");
    if (spec->L < 5 || spec->L > 1024) return elp_fail(ELP_ERR_ARG, "box edge L=%d out of range [5,1024]", spec->L);
    if (spec->linear != 0 && spec->linear != 1) return elp_fail(ELP_ERR_ARG, "linear must be 0 or 1");
    if (spec->linear && spec->kernel == 1)
        return elp_fail(ELP_ERR_ARG, "linear chains run on the specialised kernels only");
    // run lengths are 16-bit: a ring spans two sites at least, a linear chain may sit on one
    if (spec->linear && spec->N > ELP_MAX_N - 1)
        return elp_fail(ELP_ERR_ARG, "linear chain length N=%d above %d", spec->N, ELP_MAX_N - 1);
    if (spec->N < 3 || spec->N > ELP_MAX_N)
        return elp_fail(ELP_ERR_ARG, "ring length N=%d outside [3,%d]", spec->N, ELP_MAX_N);
    int p = spec->P > 0 ? spec->P : elp_get_npol(spec->density, spec->N, (long)spec->L * spec->L * spec->L);
    if (p < 1) p = 1;
    if ((long)p >= (1L << 27)) return elp_fail(ELP_ERR_ARG, "too many rings (%d)", p);
    if (2.0 * p > (double)spec->L * spec->L * spec->L)
        return elp_fail(ELP_ERR_ARG, "%d rings need at least %d sites (L=%d)", p, 2 * p, spec->L);
    memset(g, 0, sizeof(*g));
    if (!pick_geometry(spec, g))
        return elp_fail(ELP_ERR_ARG, "no valid domain geometry for L=%d (periodic=%d tile=%dx%dx%d ncol=%d)", spec->L,
                        spec->periodic, spec->tile[0], spec->tile[1], spec->tile[2], spec->ncol);
    *P = p;
    return ELP_OK;
}

elp_status elp_device_errors(const uint32_t* d_flags, cudaStream_t s)
{
    uint32_t flags = 0;
    ELP_CUDA_TRY(cudaMemcpyAsync(&flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    if (flags & 1u)
        return elp_fail(ELP_ERR_STATE, "a domain held more monomer-0 runs than its label table; steps after the "
                                       "overflow are incomplete (use the generic kernel for this melt)");
    if (flags & 4u)
        return elp_fail(ELP_ERR_STATE, "a tiled launch of several steps gave up waiting at its grid barrier; steps "
                                       "after it are incomplete");
    return ELP_OK;
}

void elp_walk_bufs_free(elp_walk_bufs* b)
{
    cudaFree(b->d_start); cudaFree(b->d_bonds); cudaFree(b->d_status); cudaFree(b->d_visit); cudaFree(b->d_cnt);
    cudaFree(b->d_obs); cudaFree(b->d_rank); cudaFree(b->d_total);
    cudaFreeHost(b->h_status); cudaFreeHost(b->h_cnt);
    *b = elp_walk_bufs();
}

elp_status elp_walk_bufs_reserve(elp_walk_bufs* b, int P, int N, size_t sites)
{
    if ((size_t)P > b->cap_rings) {
        cudaFree(b->d_start); cudaFree(b->d_status);
        b->d_start = nullptr; b->d_status = nullptr;
        ELP_CUDA_TRY(cudaMalloc((void**)&b->d_start, (size_t)P * 3 * sizeof(int32_t)));
        ELP_CUDA_TRY(cudaMalloc((void**)&b->d_status, (size_t)P * sizeof(int32_t)));
        b->bytes += (size_t)P * 16 - b->cap_rings * 16;
        b->cap_rings = (size_t)P;
    }
    if ((size_t)P * N > b->cap_bonds) {
        cudaFree(b->d_bonds);
        b->d_bonds = nullptr;
        ELP_CUDA_TRY(cudaMalloc((void**)&b->d_bonds, (size_t)P * N));
        b->bytes += (size_t)P * N - b->cap_bonds;
        b->cap_bonds = (size_t)P * N;
    }
    if (sites > b->cap_sites) {
        cudaFree(b->d_visit);
        b->d_visit = nullptr;
        ELP_CUDA_TRY(cudaMalloc((void**)&b->d_visit, sites * sizeof(uint32_t)));
        b->bytes += (sites - b->cap_sites) * 4;
        b->cap_sites = sites;
    }
    if (!b->d_cnt) ELP_CUDA_TRY(cudaMalloc((void**)&b->d_cnt, 8 * sizeof(unsigned long long)));
    return ELP_OK;
}

// Pinned host copy of the chain statuses (the copy runs behind the kernels).
static elp_status reserve_host_status(elp_walk_bufs* b, int P)
{
    if ((size_t)P > b->cap_h_rings) {
        cudaFreeHost(b->h_status);
        b->h_status = nullptr;
        b->cap_h_rings = 0;
        ELP_CUDA_TRY(cudaMallocHost((void**)&b->h_status, (size_t)P * sizeof(int32_t)));
        b->cap_h_rings = (size_t)P;
    }
    return ELP_OK;
}

elp_status elp_fetch_rings(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                           int32_t* start, uint8_t* bonds, cudaStream_t s)
{
    elp_status st = elp_walk_bufs_reserve(b, P, N, 0);
    if (st || (st = reserve_host_status(b, P))) return st;
    // list ranking: every run at once, ceil(log2 N) rounds; the chain walk
    // (one ring's latency) for boxes too large for its scratch
    const cudaError_t re = elp_rank_chains(lat, rec, L, N, P, linear, b, s);
    if (re == cudaErrorNotSupported) {
        WalkArgs w;
        memset(&w, 0, sizeof(w));
        w.lat = lat; w.rec = rec; w.L = L; w.N = N; w.P = P; w.linear = linear;
        w.start = b->d_start; w.bonds = b->d_bonds; w.status = b->d_status;
        ELP_CUDA_TRY(elp_launch_walk(&w, s));
    } else {
        ELP_CUDA_TRY(re);
    }
    ELP_CUDA_TRY(cudaMemcpyAsync(start, b->d_start, (size_t)P * 3 * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(bonds, b->d_bonds, (size_t)P * N, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(b->h_status, b->d_status, (size_t)P * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    for (int p = 0; p < P; p++)
        if (b->h_status[p])
            return elp_fail(ELP_ERR_INTEGRITY, "chain %d is broken (code %d)", p, b->h_status[p]);
    return ELP_OK;
}

elp_status elp_fetch_checked_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear,
                                  elp_walk_bufs* b, int32_t* start, uint8_t* bonds, int32_t* code, cudaStream_t s)
{
    const size_t S = (size_t)L * L * L;
    elp_status st = elp_walk_bufs_reserve(b, P, N, S);
    if (st) return st;
    if ((st = reserve_host_status(b, P))) return st;
    if (!b->h_cnt) ELP_CUDA_TRY(cudaMallocHost((void**)&b->h_cnt, 8 * sizeof(unsigned long long)));
    ELP_CUDA_TRY(cudaMemsetAsync(b->d_visit, 0, S * sizeof(uint32_t), s));
    ELP_CUDA_TRY(cudaMemsetAsync(b->d_cnt, 0, 8 * sizeof(unsigned long long), s));
    WalkArgs w;
    memset(&w, 0, sizeof(w));
    w.lat = lat; w.rec = rec; w.L = L; w.N = N; w.P = P; w.linear = linear;
    w.start = b->d_start; w.bonds = b->d_bonds; w.status = b->d_status; w.visit = b->d_visit; w.counters = b->d_cnt;
    ELP_CUDA_TRY(elp_launch_walk(&w, s));
    ELP_CUDA_TRY(elp_launch_scan(&w, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(start, b->d_start, (size_t)P * 3 * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(bonds, b->d_bonds, (size_t)P * N, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(b->h_status, b->d_status, (size_t)P * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(b->h_cnt, b->d_cnt, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    int rc = 0;
    for (int p = 0; p < P && !rc; p++)
        if (b->h_status[p]) rc = 4;
    const unsigned long long* cnt = b->h_cnt;
    if (!rc && cnt[4]) rc = 3;
    if (!rc && (cnt[0] != cnt[1] || cnt[2] != (unsigned long long)N * P || cnt[3])) rc = 4;
    *code = rc;
    return ELP_OK;
}

elp_status elp_check_melt(const uint32_t* lat, const uint32_t* rec, int L, int N, int P, int linear, elp_walk_bufs* b,
                          int32_t* code, cudaStream_t s)
{
    size_t S = (size_t)L * L * L;
    elp_status st = elp_walk_bufs_reserve(b, P, N, S);
    if (st) return st;
    ELP_CUDA_TRY(cudaMemsetAsync(b->d_visit, 0, S * sizeof(uint32_t), s));
    ELP_CUDA_TRY(cudaMemsetAsync(b->d_cnt, 0, 8 * sizeof(unsigned long long), s));
    WalkArgs w;
    memset(&w, 0, sizeof(w));
    w.lat = lat; w.rec = rec; w.L = L; w.N = N; w.P = P; w.linear = linear;
    w.status = b->d_status; w.visit = b->d_visit; w.counters = b->d_cnt;
    ELP_CUDA_TRY(elp_launch_walk(&w, s));
    ELP_CUDA_TRY(elp_launch_scan(&w, s));
    std::vector<int32_t> status((size_t)P);
    unsigned long long cnt[8];
    ELP_CUDA_TRY(cudaMemcpyAsync(status.data(), b->d_status, (size_t)P * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(cnt, b->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    int rc = 0;
    for (int p = 0; p < P && !rc; p++)
        if (status[(size_t)p]) rc = 4;
    if (!rc && cnt[4]) rc = 3;
    if (!rc && (cnt[0] != cnt[1] || cnt[2] != (unsigned long long)N * P || cnt[3])) rc = 4;
    *code = rc;
    return ELP_OK;
}

elp_status elp_read_file(const char* path, char** text, size_t* len)
{
    FILE* f = fopen(path, "rb");
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s", path);
    std::vector<char> buf;
    char chunk[1 << 16];
    size_t r;
    while ((r = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
    fclose(f);
    char* t = (char*)malloc(buf.size() + 1);
    if (!t) return elp_fail(ELP_ERR_NOMEM, "host allocation failed");
    if (!buf.empty()) memcpy(t, buf.data(), buf.size());
    t[buf.size()] = '\0';
    *text = t;
    *len = buf.size();
    return ELP_OK;
}

// ReadLatticeFile (cpupol/efpol_io.c:3-47): header then P blocks
// "len= N  t u v  <N hex digits>".
elp_status elp_parse_tuv(const char* q, const char* name, int L, int N, int P, int32_t* start, uint8_t* bonds)
{
    int lt, lu, lv, np, ml, off = 0;
    if (sscanf(q, " LT= %d LU= %d LV= %d np= %d maxPolLength= %d%n", &lt, &lu, &lv, &np, &ml, &off) != 5)
        return elp_fail(ELP_ERR_FORMAT, "%s: bad TUV header", name);
    if (lt != L || lu != L || lv != L || np != P || ml != N)
        return elp_fail(ELP_ERR_FORMAT, "%s: box %dx%dx%d np=%d N=%d does not match the job (L=%d P=%d N=%d)", name, lt,
                        lu, lv, np, ml, L, P, N);
    q += off;
    for (int p = 0; p < P; p++) {
        int len, t, u, v, k = 0;
        if (sscanf(q, " len= %d %d %d %d%n", &len, &t, &u, &v, &k) != 4 || len != N)
            return elp_fail(ELP_ERR_FORMAT, "%s: bad header of ring %d", name, p);
        q += k;
        while (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n') q++;
        for (int m = 0; m < N; m++) {
            char ch = q[m];
            int h = (ch >= '0' && ch <= '9') ? ch - '0' : (ch >= 'a' && ch <= 'f') ? ch - 'a' + 10 : -1;
            if (h < 0) return elp_fail(ELP_ERR_FORMAT, "%s: bad bond string of ring %d", name, p);
            bonds[(size_t)p * N + m] = (uint8_t)h;
        }
        q += N;
        if (*q && *q != '\n' && *q != '\r' && *q != ' ')
            return elp_fail(ELP_ERR_FORMAT, "%s: ring %d longer than %d", name, p, N);
        start[3 * (size_t)p] = t; start[3 * (size_t)p + 1] = u; start[3 * (size_t)p + 2] = v;
    }
    return ELP_OK;
}

// ---- TUV text (cpupol/efpol_io.c:50-77) ------------------------------------
extern "C" elp_status elp_format_tuv(int32_t L, int32_t N, int32_t P, const int32_t* start, const uint8_t* bonds,
                                     char* buf, size_t cap, size_t* len)
{
    if (!start || !bonds || !len || N < 1 || P < 0) return elp_fail(ELP_ERR_ARG, "bad argument");
    static const char hexd[] = "0123456789abcdef";
    char head[160];
    size_t n = 0;
    int k = snprintf(head, sizeof(head), "LT= %d\nLU= %d\nLV= %d\nnp= %d\nmaxPolLength= %d\n", L, L, L, P, N);
    if (buf) {
        if ((size_t)k >= cap) return elp_fail(ELP_ERR_ARG, "buffer too small");
        memcpy(buf, head, (size_t)k);
    }
    n += (size_t)k;
    for (int p = 0; p < P; p++) {
        k = snprintf(head, sizeof(head), "len= %d\n%u  %u  %u\t", N, (unsigned)start[3 * p], (unsigned)start[3 * p + 1],
                     (unsigned)start[3 * p + 2]);
        if (buf) {
            if (n + (size_t)k + (size_t)N + 2 > cap) return elp_fail(ELP_ERR_ARG, "buffer too small");
            memcpy(buf + n, head, (size_t)k);
            const uint8_t* b = bonds + (size_t)p * N;
            char* o = buf + n + k;
            for (int m = 0; m < N; m++) o[m] = hexd[b[m] & 15];
            o[N] = '\n';
        }
        n += (size_t)k + (size_t)N + 1;
    }
    if (buf) buf[n] = '\0';
    *len = n;
    return ELP_OK;
}

extern "C" elp_status elp_transition_table(uint8_t out[4096])
{
    if (!out) return elp_fail(ELP_ERR_ARG, "null argument");
    elp_build_table(out);
    return ELP_OK;
}
