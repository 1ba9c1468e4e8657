// elp_api.cu -- the C ABI (include/elp.h): contexts, loading, running,
// fetching, TUV files and integrity checks for one melt on one GPU.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/elp.h"
#include "elp_internal.h"
#include "elp_kernels.h"

static thread_local std::string g_last_error;

static elp_status fail(elp_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

#define CUDA_TRY(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? ELP_ERR_NOMEM : ELP_ERR_CUDA,        \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);  \
    } while (0)

struct elp_ctx {
    elp_geometry g;
    elp_smem_layout lay;
    int N, P;
    uint32_t seed, salt;
    uint64_t step;
    int device;
    int spl;                       // steps per launch (whole-box domains)
    int domains, threads;
    int nsm;                       // SMs of the device
    int generic;                   // force the generic kernel
    cudaStream_t stream;
    cudaEvent_t ev0, ev1;
    uint32_t* d_lat;
    uint32_t* d_rec;
    uint32_t* d_table;
    unsigned long long* d_acc;
    unsigned long long* d_cnt;     // 5 counters for checks
    int32_t* d_status;
    int32_t* d_start;
    uint8_t* d_bonds;
    uint32_t* d_visit;
    size_t device_bytes;
    int loaded;
};

// Device-side error flags (set by kernels instead of trapping); read after a
// stream synchronisation.
static elp_status device_errors(elp_ctx* c)
{
    uint32_t flags = 0;
    CUDA_TRY(cudaMemcpyAsync(&flags, c->d_acc + 1, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (flags & 1u)
        return fail(ELP_ERR_STATE, "a domain held more monomer-0 runs than its label table; steps after the "
                                   "overflow are incomplete (use the generic kernel for this melt)");
    return ELP_OK;
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
    int first = 0;
    if (L == 128) first = 2;  // 128 domains of 32x32x16 rather than 64 of 32^3
    for (size_t i = (size_t)first; i < sizeof(cand) / sizeof(cand[0]); i++) {
        g->tx = cand[i][0]; g->ty = cand[i][1]; g->tz = cand[i][2];
        if (L % g->tx || L % g->ty || L % g->tz) continue;
        g->ncol = s->ncol > 0 ? s->ncol : elp_pick_ncol(g->tx);
        if (g->ncol && elp_geometry_ok(g)) return 1;
    }
    return 0;
}

extern "C" elp_status elp_create(const elp_job_spec* spec, elp_ctx** out)
{
    if (!spec || !out) return fail(ELP_ERR_ARG, "null argument");
    *out = nullptr;
    if (spec->L < 5 || spec->L > 1024) return fail(ELP_ERR_ARG, "box edge L=%d out of range [5,1024]", spec->L);
    if (spec->N < 3 || spec->N > ELP_MAX_N) return fail(ELP_ERR_ARG, "ring length N=%d outside [3,%d]", spec->N, ELP_MAX_N);
    int P = spec->P > 0 ? spec->P : elp_get_npol(spec->density, spec->N, (long)spec->L * spec->L * spec->L);
    if (P < 1) P = 1;
    if ((long)P >= (1L << 27)) return fail(ELP_ERR_ARG, "too many rings (%d)", P);
    elp_geometry g;
    memset(&g, 0, sizeof(g));
    if (!pick_geometry(spec, &g))
        return fail(ELP_ERR_ARG, "no valid domain geometry for L=%d (periodic=%d tile=%dx%dx%d ncol=%d)", spec->L,
                    spec->periodic, spec->tile[0], spec->tile[1], spec->tile[2], spec->ncol);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(ELP_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (spec->device < 0 || spec->device >= ndev) return fail(ELP_ERR_ARG, "device %d not present", spec->device);
    CUDA_TRY(cudaSetDevice(spec->device));

    elp_ctx* c = (elp_ctx*)calloc(1, sizeof(elp_ctx));
    if (!c) return fail(ELP_ERR_NOMEM, "host allocation failed");
    c->g = g;
    elp_layout(&g, &c->lay);
    c->N = spec->N;
    c->P = P;
    c->seed = spec->seed;
    c->salt = spec->salt;
    c->device = spec->device;
    c->spl = spec->steps_per_launch > 0 ? spec->steps_per_launch : 1;
    c->generic = spec->kernel == 1;
    if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, spec->device) != cudaSuccess || c->nsm < 1)
        c->nsm = 148;
    c->domains = g.periodic ? 1 : (g.L / g.tx) * (g.L / g.ty) * (g.L / g.tz);
    c->threads = (c->lay.groups + 31) / 32 * 32;
    if (c->threads < 32) c->threads = 32;

    size_t S = (size_t)g.L * g.L * g.L;
    elp_status st = ELP_OK;
#define ALLOC(ptr, bytes)                                                                         \
    do {                                                                                          \
        cudaError_t ea_ = cudaMalloc((void**)&(ptr), (bytes));                                    \
        if (ea_ != cudaSuccess) { st = fail(ELP_ERR_NOMEM, "cudaMalloc(%zu): %s", (size_t)(bytes), \
                                             cudaGetErrorString(ea_)); goto bad; }                \
        c->device_bytes += (bytes);                                                               \
    } while (0)
    ALLOC(c->d_lat, S * sizeof(uint32_t));
    ALLOC(c->d_rec, (size_t)P * ELP_REC_WORDS * sizeof(uint32_t));
    ALLOC(c->d_table, 4096);
    ALLOC(c->d_acc, 8 * sizeof(unsigned long long));
    ALLOC(c->d_cnt, 8 * sizeof(unsigned long long));
    ALLOC(c->d_status, (size_t)P * sizeof(int32_t));
#undef ALLOC
    {
        uint8_t tab[4096];
        elp_build_table(tab);
        if (cudaMemcpy(c->d_table, tab, 4096, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(c->d_lat, 0, S * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemset(c->d_acc, 0, 8 * sizeof(unsigned long long)) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
            st = fail(ELP_ERR_CUDA, "context set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
            goto bad;
        }
    }
    *out = c;
    return ELP_OK;
bad:
    elp_destroy(c);
    return st;
}

extern "C" void elp_destroy(elp_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_lat); cudaFree(c->d_rec); cudaFree(c->d_table); cudaFree(c->d_acc); cudaFree(c->d_cnt);
    cudaFree(c->d_status); cudaFree(c->d_start); cudaFree(c->d_bonds); cudaFree(c->d_visit);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    free(c);
}

static elp_status upload(elp_ctx* c, const uint32_t* lat, const uint32_t* rec, uint64_t step)
{
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaMemcpyAsync(c->d_lat, lat, S * 4, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_rec, rec, (size_t)c->P * ELP_REC_WORDS * 4, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->step = step;
    c->loaded = 1;
    return ELP_OK;
}

extern "C" elp_status elp_load_chains(elp_ctx* c, const int32_t* start, const uint8_t* bonds, uint64_t step)
{
    if (!c || !start || !bonds) return fail(ELP_ERR_ARG, "null argument");
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    std::vector<uint32_t> lat(S), rec((size_t)c->P * ELP_REC_WORDS);
    int rc = elp_chains_to_sites(c->g.L, c->N, c->P, start, bonds, lat.data(), rec.data());
    if (rc == 3) return fail(ELP_ERR_INTEGRITY, "two rings or two runs of a ring share a site (code 3)");
    if (rc) return fail(ELP_ERR_INTEGRITY, "invalid ring: bad bond, not closed, or on a single site (code 4)");
    return upload(c, lat.data(), rec.data(), step);
}

extern "C" elp_status elp_init_melt(elp_ctx* c)
{
    if (!c) return fail(ELP_ERR_ARG, "null context");
    std::vector<int32_t> start((size_t)c->P * 3);
    std::vector<uint8_t> bonds((size_t)c->P * c->N);
    if (elp_initial_chains(c->g.L, c->N, c->P, start.data(), bonds.data()))
        return fail(ELP_ERR_ARG, "initial grid cannot hold %d rings of %d in L=%d", c->P, c->N, c->g.L);
    return elp_load_chains(c, start.data(), bonds.data(), 0);
}

extern "C" elp_status elp_set_state(elp_ctx* c, const uint32_t* words, const uint32_t* records, uint64_t step)
{
    if (!c || !words || !records) return fail(ELP_ERR_ARG, "null argument");
    return upload(c, words, records, step);
}

extern "C" elp_status elp_get_state(elp_ctx* c, uint32_t* words, uint32_t* records)
{
    if (!c || !words || !records) return fail(ELP_ERR_ARG, "null argument");
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaMemcpyAsync(words, c->d_lat, S * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(records, c->d_rec, (size_t)c->P * ELP_REC_WORDS * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return device_errors(c);
}

static elp_status enqueue_steps(elp_ctx* c, int64_t nsteps)
{
    SweepArgs a;
    a.lat = c->d_lat;
    a.rec = c->d_rec;
    a.table = c->d_table;
    a.accepted = c->d_acc;
    a.error = reinterpret_cast<uint32_t*>(c->d_acc + 1);
    a.nchains = c->P;
    a.L = c->g.L;
    a.periodic = c->g.periodic;
    a.tx = c->g.tx; a.ty = c->g.ty; a.tz = c->g.tz;
    a.ncol = c->g.ncol;
    a.sx = c->lay.sx; a.sxy = c->lay.sxy; a.ox = c->lay.ox;
    a.words = c->lay.words;
    a.groups = c->lay.groups;
    a.seed = c->seed;
    a.salt = c->salt;
    while (nsteps > 0) {
        int k = c->g.periodic ? (int)(nsteps < c->spl ? nsteps : c->spl) : 1;
        a.step0 = c->step;
        a.nsteps = k;
        cudaError_t e = c->generic ? cudaErrorNotSupported : elp_launch_sweep2(&a, c->nsm, c->stream);
        if (e == cudaErrorNotSupported) e = elp_launch_sweep(&a, c->domains, c->threads, c->lay.bytes, c->stream);
        CUDA_TRY(e);
        c->step += (uint64_t)k;
        nsteps -= k;
    }
    return ELP_OK;
}

extern "C" elp_status elp_run(elp_ctx* c, int64_t nsteps)
{
    if (!c) return fail(ELP_ERR_ARG, "null context");
    if (!c->loaded) return fail(ELP_ERR_STATE, "no configuration loaded");
    if (nsteps < 0) return fail(ELP_ERR_ARG, "negative step count");
    CUDA_TRY(cudaSetDevice(c->device));
    return enqueue_steps(c, nsteps);
}

extern "C" elp_status elp_run_timed(elp_ctx* c, int64_t nsteps, float* ms)
{
    if (!c || !ms) return fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return fail(ELP_ERR_STATE, "no configuration loaded");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
    elp_status st = enqueue_steps(c, nsteps);
    if (st) return st;
    CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(cudaEventSynchronize(c->ev1));
    CUDA_TRY(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return device_errors(c);
}

extern "C" elp_status elp_sync(elp_ctx* c)
{
    if (!c) return fail(ELP_ERR_ARG, "null context");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return device_errors(c);
}

extern "C" elp_status elp_accepted(elp_ctx* c, uint64_t* acc)
{
    if (!c || !acc) return fail(ELP_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    unsigned long long v = 0;
    CUDA_TRY(cudaMemcpyAsync(&v, c->d_acc, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    *acc = v;
    return ELP_OK;
}

static elp_status ensure_chain_buffers(elp_ctx* c)
{
    if (!c->d_start) {
        CUDA_TRY(cudaMalloc((void**)&c->d_start, (size_t)c->P * 3 * sizeof(int32_t)));
        c->device_bytes += (size_t)c->P * 3 * sizeof(int32_t);
    }
    if (!c->d_bonds) {
        CUDA_TRY(cudaMalloc((void**)&c->d_bonds, (size_t)c->P * c->N));
        c->device_bytes += (size_t)c->P * c->N;
    }
    return ELP_OK;
}

extern "C" elp_status elp_fetch_chains(elp_ctx* c, int32_t* start, uint8_t* bonds)
{
    if (!c || !start || !bonds) return fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return fail(ELP_ERR_STATE, "no configuration loaded");
    CUDA_TRY(cudaSetDevice(c->device));
    elp_status st = ensure_chain_buffers(c);
    if (st) return st;
    WalkArgs w;
    memset(&w, 0, sizeof(w));
    w.lat = c->d_lat; w.rec = c->d_rec; w.L = c->g.L; w.N = c->N; w.P = c->P;
    w.start = c->d_start; w.bonds = c->d_bonds; w.status = c->d_status;
    CUDA_TRY(elp_launch_walk(&w, c->stream));
    std::vector<int32_t> status((size_t)c->P);
    CUDA_TRY(cudaMemcpyAsync(start, c->d_start, (size_t)c->P * 3 * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(bonds, c->d_bonds, (size_t)c->P * c->N, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(status.data(), c->d_status, (size_t)c->P * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    elp_status dev = device_errors(c);
    if (dev) return dev;
    for (int p = 0; p < c->P; p++)
        if (status[(size_t)p]) return fail(ELP_ERR_INTEGRITY, "ring %d cannot be walked (code %d)", p, status[(size_t)p]);
    return ELP_OK;
}

extern "C" elp_status elp_check(elp_ctx* c, int32_t* code)
{
    if (!c || !code) return fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return fail(ELP_ERR_STATE, "no configuration loaded");
    CUDA_TRY(cudaSetDevice(c->device));
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    if (!c->d_visit) {
        CUDA_TRY(cudaMalloc((void**)&c->d_visit, S * sizeof(uint32_t)));
        c->device_bytes += S * sizeof(uint32_t);
    }
    CUDA_TRY(cudaMemsetAsync(c->d_visit, 0, S * sizeof(uint32_t), c->stream));
    CUDA_TRY(cudaMemsetAsync(c->d_cnt, 0, 8 * sizeof(unsigned long long), c->stream));
    WalkArgs w;
    memset(&w, 0, sizeof(w));
    w.lat = c->d_lat; w.rec = c->d_rec; w.L = c->g.L; w.N = c->N; w.P = c->P;
    w.status = c->d_status; w.visit = c->d_visit; w.counters = c->d_cnt;
    CUDA_TRY(elp_launch_walk(&w, c->stream));
    CUDA_TRY(elp_launch_scan(&w, c->stream));
    std::vector<int32_t> status((size_t)c->P);
    unsigned long long cnt[8];
    CUDA_TRY(cudaMemcpyAsync(status.data(), c->d_status, (size_t)c->P * 4, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(cnt, c->d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    elp_status dev = device_errors(c);
    if (dev) return dev;
    int rc = 0;
    for (int p = 0; p < c->P && !rc; p++)
        if (status[(size_t)p]) rc = 4;
    if (!rc && cnt[4]) rc = 3;
    if (!rc && (cnt[0] != cnt[1] || cnt[2] != (unsigned long long)c->N * c->P || cnt[3])) rc = 4;
    *code = rc;
    return ELP_OK;
}

extern "C" elp_status elp_get_info(const elp_ctx* c, elp_info* info)
{
    if (!c || !info) return fail(ELP_ERR_ARG, "null argument");
    info->L = c->g.L; info->N = c->N; info->P = c->P;
    info->periodic = c->g.periodic;
    info->tile[0] = c->g.tx; info->tile[1] = c->g.ty; info->tile[2] = c->g.tz;
    info->ncol = c->g.ncol;
    info->domains = c->domains;
    info->threads = c->threads;
    info->smem_bytes = c->lay.bytes;
    info->step = c->step;
    info->device_bytes = c->device_bytes;
    return ELP_OK;
}

extern "C" elp_status elp_transition_table(uint8_t out[4096])
{
    if (!out) return fail(ELP_ERR_ARG, "null argument");
    elp_build_table(out);
    return ELP_OK;
}

// ---- TUV text (cpupol/efpol_io.c:50-77) ------------------------------------
extern "C" elp_status elp_format_tuv(int32_t L, int32_t N, int32_t P, const int32_t* start, const uint8_t* bonds,
                                     char* buf, size_t cap, size_t* len)
{
    if (!start || !bonds || !len || N < 1 || P < 0) return fail(ELP_ERR_ARG, "bad argument");
    static const char hexd[] = "0123456789abcdef";
    char head[160];
    size_t n = 0;
    int k = snprintf(head, sizeof(head), "LT= %d\nLU= %d\nLV= %d\nnp= %d\nmaxPolLength= %d\n", L, L, L, P, N);
    if (buf) {
        if ((size_t)k >= cap) return fail(ELP_ERR_ARG, "buffer too small");
        memcpy(buf, head, (size_t)k);
    }
    n += (size_t)k;
    for (int p = 0; p < P; p++) {
        k = snprintf(head, sizeof(head), "len= %d\n%u  %u  %u\t", N, (unsigned)start[3 * p], (unsigned)start[3 * p + 1],
                     (unsigned)start[3 * p + 2]);
        if (buf) {
            if (n + (size_t)k + (size_t)N + 2 > cap) return fail(ELP_ERR_ARG, "buffer too small");
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

extern "C" elp_status elp_write_tuv(elp_ctx* c, const char* path)
{
    if (!c || !path) return fail(ELP_ERR_ARG, "null argument");
    std::vector<int32_t> start((size_t)c->P * 3);
    std::vector<uint8_t> bonds((size_t)c->P * c->N);
    elp_status st = elp_fetch_chains(c, start.data(), bonds.data());
    if (st) return st;
    size_t len = 0;
    elp_format_tuv(c->g.L, c->N, c->P, start.data(), bonds.data(), nullptr, 0, &len);
    std::vector<char> text(len + 1);
    st = elp_format_tuv(c->g.L, c->N, c->P, start.data(), bonds.data(), text.data(), len + 1, &len);
    if (st) return st;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(ELP_ERR_IO, "cannot open %s for writing", path);
    size_t wr = fwrite(text.data(), 1, len, f);
    int cl = fclose(f);
    if (wr != len || cl) return fail(ELP_ERR_IO, "short write to %s", path);
    return ELP_OK;
}

// ReadLatticeFile (cpupol/efpol_io.c:3-47): header then P blocks
// "len= N  t u v  <N hex digits>".
extern "C" elp_status elp_load_tuv(elp_ctx* c, const char* path, uint64_t step)
{
    if (!c || !path) return fail(ELP_ERR_ARG, "null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(ELP_ERR_IO, "cannot open %s", path);
    std::vector<char> text;
    char chunk[1 << 16];
    size_t r;
    while ((r = fread(chunk, 1, sizeof(chunk), f)) > 0) text.insert(text.end(), chunk, chunk + r);
    fclose(f);
    text.push_back('\0');
    const char* q = text.data();
    int lt, lu, lv, np, ml, off = 0;
    if (sscanf(q, " LT= %d LU= %d LV= %d np= %d maxPolLength= %d%n", &lt, &lu, &lv, &np, &ml, &off) != 5)
        return fail(ELP_ERR_FORMAT, "%s: bad TUV header", path);
    if (lt != c->g.L || lu != c->g.L || lv != c->g.L || np != c->P || ml != c->N)
        return fail(ELP_ERR_FORMAT, "%s: box %dx%dx%d np=%d N=%d does not match the job (L=%d P=%d N=%d)", path, lt, lu, lv,
                    np, ml, c->g.L, c->P, c->N);
    q += off;
    std::vector<int32_t> start((size_t)c->P * 3);
    std::vector<uint8_t> bonds((size_t)c->P * c->N);
    for (int p = 0; p < c->P; p++) {
        int len, t, u, v, k = 0;
        if (sscanf(q, " len= %d %d %d %d%n", &len, &t, &u, &v, &k) != 4 || len != c->N)
            return fail(ELP_ERR_FORMAT, "%s: bad header of ring %d", path, p);
        q += k;
        while (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n') q++;
        for (int m = 0; m < c->N; m++) {
            char ch = q[m];
            int h = (ch >= '0' && ch <= '9') ? ch - '0' : (ch >= 'a' && ch <= 'f') ? ch - 'a' + 10 : -1;
            if (h < 0) return fail(ELP_ERR_FORMAT, "%s: bad bond string of ring %d", path, p);
            bonds[(size_t)p * c->N + m] = (uint8_t)h;
        }
        q += c->N;
        if (*q && *q != '\n' && *q != '\r' && *q != ' ') return fail(ELP_ERR_FORMAT, "%s: ring %d too long", path, p);
        start[3 * (size_t)p] = t; start[3 * (size_t)p + 1] = u; start[3 * (size_t)p + 2] = v;
    }
    return elp_load_chains(c, start.data(), bonds.data(), step);
}

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

extern "C" const char* elp_last_error(void) { return g_last_error.c_str(); }
