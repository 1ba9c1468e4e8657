// elp_batch.cu -- the batched engine: many independent melts (replicas,
// seeds, parameter sweeps) of uneven box size and ring length advanced
// together on one GPU.
//
// All lattices and chain records live in one packed ragged arena.  Melts with
// the same domain geometry form a group (elp_group.h) that one kernel launch
// serves: whole-box melts (L <= 32) run many steps per launch without leaving
// shared memory; tiled melts run one step per launch, replayed from a CUDA
// graph.  Every group has its own stream, so groups of different shapes run
// concurrently.  A melt gives the same bits in a batch as alone (same kernel,
// same counters).
#include <cuda_runtime.h>
#include <string.h>

#include <map>
#include <new>
#include <tuple>
#include <algorithm>
#include <vector>

#include "elp_common.h"
#include "elp_group.h"
#include "elp_kernels.h"

namespace {
struct Member {
    int group, index;          // group and position inside it
    elp_geometry g;
    int N, P;
    int linear;                // 1: linear chains
    uint32_t seed, salt;
    uint32_t* lat;
    uint32_t* rec;
    unsigned long long* acc;
    int loaded;
};
}  // namespace

struct elp_batch {
    int device = 0, nsm = 148;
    std::vector<Member> m;
    std::vector<elp_group*> groups;
    std::vector<cudaStream_t> streams;
    cudaStream_t main = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> done;
    uint32_t* d_lat = nullptr;
    uint32_t* d_rec = nullptr;
    unsigned long long* d_acc = nullptr;   // one per melt
    uint32_t* d_err = nullptr;             // one per group
    uint32_t* d_table = nullptr;
    size_t device_bytes = 0;
    elp_walk_bufs wb;
};

extern "C" void elp_batch_destroy(elp_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    for (cudaStream_t s : b->streams) cudaStreamSynchronize(s);
    for (elp_group* G : b->groups) {
        elp_group_free(G);
        delete G;
    }
    elp_walk_bufs_free(&b->wb);
    for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->done) cudaEventDestroy(e);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->main) cudaStreamDestroy(b->main);
    cudaFree(b->d_lat); cudaFree(b->d_rec); cudaFree(b->d_acc); cudaFree(b->d_err); cudaFree(b->d_table);
    delete b;
}

extern "C" elp_status elp_batch_create(const elp_job_spec* specs, int32_t njobs, int32_t device, elp_batch** out)
{
    if (!specs || !out || njobs < 1) return elp_fail(ELP_ERR_ARG, "bad argument");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return elp_fail(ELP_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return elp_fail(ELP_ERR_ARG, "device %d not present", device);
    ELP_CUDA_TRY(cudaSetDevice(device));
    elp_batch* b = new (std::nothrow) elp_batch();
    if (!b) return elp_fail(ELP_ERR_NOMEM, "host allocation failed");
    b->device = device;
    if (cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || b->nsm < 1) b->nsm = 148;

    // resolve every melt; group by geometry, steps per launch and kernel choice
    std::map<std::tuple<int, int, int, int, int, int, int, int, int>, int> key2g;
    std::vector<std::tuple<elp_geometry, int, int>> gdesc;  // geometry, spl, generic
    size_t lat_words = 0, rec_words = 0;
    elp_status st = ELP_OK;
    for (int j = 0; j < njobs; j++) {
        Member mm;
        memset(&mm, 0, sizeof(mm));
        st = elp_resolve_spec(&specs[j], &mm.P, &mm.g);
        if (st) {
            elp_batch_destroy(b);
            return elp_fail(st, "melt %d: %s", j, elp_last_error());
        }
        mm.N = specs[j].N;
        mm.linear = specs[j].linear;
        mm.seed = specs[j].seed;
        mm.salt = specs[j].salt;
        const int spl = specs[j].steps_per_launch > 0 ? specs[j].steps_per_launch : 1;
        const int gen = specs[j].kernel == 1;
        // rings and linear chains run in different groups (different kernels)
        auto key = std::make_tuple(mm.g.periodic, mm.g.L, mm.g.tx, mm.g.ty, mm.g.tz, mm.g.ncol, spl, gen, mm.linear);
        auto it = key2g.find(key);
        if (it == key2g.end()) {
            it = key2g.emplace(key, (int)gdesc.size()).first;
            gdesc.emplace_back(mm.g, spl, gen);
        }
        mm.group = it->second;
        b->m.push_back(mm);
        lat_words += ((size_t)mm.g.L * mm.g.L * mm.g.L + 63) / 64 * 64;
        rec_words += (size_t)mm.P * ELP_REC_WORDS;
    }
    // A tiled launch of several steps is cooperative: it starts only when all
    // its CTAs fit at once and then holds every SM until its last step, which
    // would serialise the groups that otherwise overlap.  With more than one
    // group, tiled groups take one step per launch (the same bits).
    if (gdesc.size() > 1)
        for (auto& gd : gdesc)
            if (!std::get<0>(gd).periodic) std::get<1>(gd) = 1;
    // one packed arena for all lattices and records
    e = cudaMalloc((void**)&b->d_lat, lat_words * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_rec, rec_words * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_acc, (size_t)njobs * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_err, gdesc.size() * sizeof(uint32_t) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_table, 4096);
    if (e != cudaSuccess) {
        elp_batch_destroy(b);
        return elp_fail(e == cudaErrorMemoryAllocation ? ELP_ERR_NOMEM : ELP_ERR_CUDA, "arena allocation failed: %s",
                        cudaGetErrorString(e));
    }
    b->device_bytes = lat_words * 4 + rec_words * 4 + (size_t)njobs * 8 + gdesc.size() * 16 + 4096;
    uint8_t tab[4096];
    elp_build_table(tab);
    if (cudaMemcpy(b->d_table, tab, 4096, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->d_lat, 0, lat_words * 4) != cudaSuccess ||
        cudaMemset(b->d_acc, 0, (size_t)njobs * 8) != cudaSuccess ||
        cudaMemset(b->d_err, 0, gdesc.size() * 16) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev0, cudaEventDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev1, cudaEventDefault) != cudaSuccess) {
        elp_batch_destroy(b);
        return elp_fail(ELP_ERR_CUDA, "batch set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    size_t lo = 0, ro = 0;
    for (size_t g = 0; g < gdesc.size(); g++) {
        cudaStream_t s;
        cudaEvent_t ev;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            elp_batch_destroy(b);
            return elp_fail(ELP_ERR_CUDA, "stream creation failed");
        }
        b->streams.push_back(s);
        b->done.push_back(ev);
        elp_group* G = new elp_group();
        b->groups.push_back(G);
        if (elp_group_init(G, std::get<0>(gdesc[g]), b->nsm, std::get<2>(gdesc[g]), std::get<1>(gdesc[g]), b->d_table,
                           b->d_err + 4 * g, s) != cudaSuccess) {
            elp_batch_destroy(b);
            return elp_fail(ELP_ERR_CUDA, "group set-up failed");
        }
    }
    for (size_t j = 0; j < b->m.size(); j++) {
        Member& mm = b->m[j];
        mm.lat = b->d_lat + lo;
        mm.rec = b->d_rec + ro;
        mm.acc = b->d_acc + j;
        lo += ((size_t)mm.g.L * mm.g.L * mm.g.L + 63) / 64 * 64;
        ro += (size_t)mm.P * ELP_REC_WORDS;
        elp_group* G = b->groups[(size_t)mm.group];
        mm.index = (int)G->jobs.size();
        elp_group_add(G, mm.lat, mm.rec, mm.acc, mm.N, mm.P, mm.seed, mm.salt, 0, mm.linear);
    }
    for (elp_group* G : b->groups) {
        if ((e = elp_group_commit(G)) != cudaSuccess) {
            elp_batch_destroy(b);
            return elp_fail(ELP_ERR_CUDA, "group commit failed: %s", cudaGetErrorString(e));
        }
    }
    for (size_t j = 0; j < b->m.size(); j++)
        if (b->m[j].linear && !b->groups[(size_t)b->m[j].group]->specialised) {
            const elp_geometry gj = b->m[j].g;
            elp_batch_destroy(b);
            return elp_fail(ELP_ERR_ARG, "melt %zu: linear chains need a domain shape with a specialised kernel "
                                         "(L=%d tile %dx%dx%d)", j, gj.L, gj.tx, gj.ty, gj.tz);
        }
    *out = b;
    return ELP_OK;
}

extern "C" int32_t elp_batch_size(const elp_batch* b) { return b ? (int32_t)b->m.size() : 0; }

static elp_status job_ok(const elp_batch* b, int32_t j)
{
    if (!b) return elp_fail(ELP_ERR_ARG, "null batch");
    if (j < 0 || (size_t)j >= b->m.size()) return elp_fail(ELP_ERR_ARG, "melt %d out of range", j);
    return ELP_OK;
}

static elp_status errors_of(elp_batch* b, int g)
{
    return elp_device_errors(b->d_err + 4 * (size_t)g, b->streams[(size_t)g]);
}

extern "C" elp_status elp_batch_load_chains(elp_batch* b, int32_t j, const int32_t* start, const uint8_t* bonds,
                                            uint64_t step)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!start || !bonds) return elp_fail(ELP_ERR_ARG, "null argument");
    Member& mm = b->m[(size_t)j];
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t s = b->streams[(size_t)mm.group];
    // built in place on the device; until that succeeds the melt holds no configuration
    mm.loaded = 0;
    st = elp_build_melt(mm.lat, mm.rec, mm.g.L, mm.N, mm.P, mm.linear, start, bonds, &b->wb, s);
    if (st) return elp_fail(st, "melt %d: %s", j, elp_last_error());
    ELP_CUDA_TRY(elp_group_set_step(b->groups[(size_t)mm.group], mm.index, step));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    mm.loaded = 1;
    return ELP_OK;
}

extern "C" elp_status elp_batch_init_melts(elp_batch* b)
{
    if (!b) return elp_fail(ELP_ERR_ARG, "null batch");
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    for (size_t j = 0; j < b->m.size(); j++) {
        Member& mm = b->m[j];
        cudaStream_t s = b->streams[(size_t)mm.group];
        mm.loaded = 0;
        elp_status st = elp_init_melt_device(mm.lat, mm.rec, mm.g.L, mm.N, mm.P, mm.linear, s);
        if (st) return elp_fail(st, "melt %zu: %s", j, elp_last_error());
        ELP_CUDA_TRY(elp_group_set_step(b->groups[(size_t)mm.group], mm.index, 0));
    }
    for (cudaStream_t s : b->streams) ELP_CUDA_TRY(cudaStreamSynchronize(s));
    for (Member& mm : b->m) mm.loaded = 1;
    return ELP_OK;
}

static elp_status enqueue(elp_batch* b, int64_t nsteps)
{
    for (const Member& mm : b->m)
        if (!mm.loaded) return elp_fail(ELP_ERR_STATE, "a melt of the batch has no configuration");
    for (elp_group* G : b->groups) ELP_CUDA_TRY(elp_group_run(G, nsteps));
    return ELP_OK;
}

extern "C" elp_status elp_batch_run(elp_batch* b, int64_t nsteps)
{
    if (!b) return elp_fail(ELP_ERR_ARG, "null batch");
    if (nsteps < 0) return elp_fail(ELP_ERR_ARG, "negative step count");
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    return enqueue(b, nsteps);
}

extern "C" elp_status elp_batch_run_timed(elp_batch* b, int64_t nsteps, float* ms)
{
    if (!b || !ms) return elp_fail(ELP_ERR_ARG, "null argument");
    if (nsteps < 0) return elp_fail(ELP_ERR_ARG, "negative step count");
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    for (cudaStream_t s : b->streams) ELP_CUDA_TRY(cudaStreamSynchronize(s));
    ELP_CUDA_TRY(cudaEventRecord(b->ev0, b->main));
    for (cudaStream_t s : b->streams) ELP_CUDA_TRY(cudaStreamWaitEvent(s, b->ev0, 0));
    elp_status st = enqueue(b, nsteps);
    if (st) return st;
    for (size_t g = 0; g < b->streams.size(); g++) {
        ELP_CUDA_TRY(cudaEventRecord(b->done[g], b->streams[g]));
        ELP_CUDA_TRY(cudaStreamWaitEvent(b->main, b->done[g], 0));
    }
    ELP_CUDA_TRY(cudaEventRecord(b->ev1, b->main));
    ELP_CUDA_TRY(cudaEventSynchronize(b->ev1));
    ELP_CUDA_TRY(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    for (size_t g = 0; g < b->groups.size(); g++) {
        st = errors_of(b, (int)g);
        if (st) return st;
    }
    return ELP_OK;
}

extern "C" elp_status elp_batch_sync(elp_batch* b)
{
    if (!b) return elp_fail(ELP_ERR_ARG, "null batch");
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    for (size_t g = 0; g < b->groups.size(); g++) {
        elp_status st = errors_of(b, (int)g);
        if (st) return st;
    }
    return ELP_OK;
}

extern "C" elp_status elp_batch_fetch_chains(elp_batch* b, int32_t j, int32_t* start, uint8_t* bonds)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!start || !bonds) return elp_fail(ELP_ERR_ARG, "null argument");
    const Member& mm = b->m[(size_t)j];
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    if ((st = errors_of(b, mm.group))) return st;
    return elp_fetch_rings(mm.lat, mm.rec, mm.g.L, mm.N, mm.P, mm.linear, &b->wb, start, bonds, b->streams[(size_t)mm.group]);
}

extern "C" elp_status elp_batch_observe(elp_batch* b, int32_t j, double* cms_tuv, double* rg2, double* sl,
                                        uint64_t* run_hist, int32_t nbins)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    const Member& mm = b->m[(size_t)j];
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    if ((st = errors_of(b, mm.group))) return st;
    return elp_observe_melt(mm.lat, mm.rec, mm.g.L, mm.N, mm.P, mm.linear, &b->wb, cms_tuv, rg2, sl, run_hist, nbins,
                            b->streams[(size_t)mm.group]);
}

extern "C" elp_status elp_batch_get_state(elp_batch* b, int32_t j, uint32_t* words, uint32_t* records)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!words || !records) return elp_fail(ELP_ERR_ARG, "null argument");
    const Member& mm = b->m[(size_t)j];
    cudaStream_t s = b->streams[(size_t)mm.group];
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    ELP_CUDA_TRY(cudaMemcpyAsync(words, mm.lat, (size_t)mm.g.L * mm.g.L * mm.g.L * 4, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaMemcpyAsync(records, mm.rec, (size_t)mm.P * ELP_REC_WORDS * 4, cudaMemcpyDeviceToHost, s));
    return errors_of(b, mm.group);
}

extern "C" elp_status elp_batch_check(elp_batch* b, int32_t j, int32_t* code)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!code) return elp_fail(ELP_ERR_ARG, "null argument");
    const Member& mm = b->m[(size_t)j];
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    if ((st = errors_of(b, mm.group))) return st;
    return elp_check_melt(mm.lat, mm.rec, mm.g.L, mm.N, mm.P, mm.linear, &b->wb, code, b->streams[(size_t)mm.group]);
}

extern "C" elp_status elp_batch_accepted(elp_batch* b, int32_t j, uint64_t* acc)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!acc) return elp_fail(ELP_ERR_ARG, "null argument");
    const Member& mm = b->m[(size_t)j];
    cudaStream_t s = b->streams[(size_t)mm.group];
    unsigned long long v = 0;
    ELP_CUDA_TRY(cudaSetDevice(b->device));
    ELP_CUDA_TRY(cudaMemcpyAsync(&v, mm.acc, 8, cudaMemcpyDeviceToHost, s));
    ELP_CUDA_TRY(cudaStreamSynchronize(s));
    *acc = v;
    return ELP_OK;
}

extern "C" elp_status elp_batch_job_info(const elp_batch* b, int32_t j, elp_info* info)
{
    elp_status st = job_ok(b, j);
    if (st) return st;
    if (!info) return elp_fail(ELP_ERR_ARG, "null argument");
    const Member& mm = b->m[(size_t)j];
    const elp_group* G = b->groups[(size_t)mm.group];
    memset(info, 0, sizeof(*info));
    info->L = mm.g.L; info->N = mm.N; info->P = mm.P;
    info->periodic = mm.g.periodic;
    info->tile[0] = mm.g.tx; info->tile[1] = mm.g.ty; info->tile[2] = mm.g.tz;
    info->ncol = mm.g.ncol;
    info->domains = mm.g.periodic ? 1 : (mm.g.L / mm.g.tx) * (mm.g.L / mm.g.ty) * (mm.g.L / mm.g.tz);
    info->threads = G->threads;
    info->specialised = G->specialised;
    info->linear = mm.linear;
    info->smem_bytes = G->smem;
    info->step = elp_group_step(G, mm.index);
    info->device_bytes = b->device_bytes + b->wb.bytes;
    info->kernels = G->kernels;   // of the member's geometry group
    return ELP_OK;
}

// ---- autotuner ---------------------------------------------------------------
// Clock factor of a candidate: 1 for the whole box, the measured time factor
// of its tile shape, 0 if that shape was not measured.
static double clock_factor(const elp_job_spec& c)
{
    return c.periodic == 1 ? 1.0 : elp_time_factor(0, c.tile[0], c.tile[1], c.tile[2]);
}

// Candidate geometries for a melt: its whole box on chip (if that fits) and
// every tile shape of the preference list that divides the box, each with a
// few steps-per-launch values.  Each is timed on `copies` copies of the initial melt
// run as one batch (the best tile depends on how many melts share the GPU).
extern "C" elp_status elp_autotune(const elp_job_spec* in, int32_t copies, int32_t steps, elp_job_spec* out,
                                   float* ms_per_step)
{
    if (!in || !out || copies < 1 || steps < 1) return elp_fail(ELP_ERR_ARG, "bad argument");
    std::vector<elp_job_spec> cand;
    {
        elp_job_spec s = *in;
        s.periodic = 1;
        s.tile[0] = s.tile[1] = s.tile[2] = 0;
        s.ncol = 0;
        int P;
        elp_geometry g;
        if (elp_resolve_spec(&s, &P, &g) == ELP_OK) {
            const int spls[] = {1, 10, 100};
            for (int spl : spls) {
                if (spl > steps) continue;
                s.steps_per_launch = spl;
                cand.push_back(s);
            }
        }
    }
    static const int tiles[][3] = {{32, 32, 32}, {48, 24, 24}, {32, 32, 16}, {24, 24, 24}, {32, 16, 16},
                                   {16, 16, 16}, {40, 20, 20}, {20, 20, 20}, {16, 16, 8}};
    for (const auto& t : tiles) {
        elp_job_spec s = *in;
        s.periodic = 0;
        s.tile[0] = t[0]; s.tile[1] = t[1]; s.tile[2] = t[2];
        s.ncol = 0;
        int P;
        elp_geometry g;
        if (in->L % t[0] || in->L % t[1] || in->L % t[2]) continue;
        if (elp_resolve_spec(&s, &P, &g) != ELP_OK) continue;
        const int spls[] = {1, 10, 100};
        for (int spl : spls) {
            if (spl > steps) continue;
            s.steps_per_launch = spl;
            cand.push_back(s);
        }
    }
    // a shape whose clock was never measured cannot be compared
    cand.erase(std::remove_if(cand.begin(), cand.end(), [](const elp_job_spec& c) { return clock_factor(c) <= 0.0; }),
               cand.end());
    if (cand.empty()) return elp_fail(ELP_ERR_ARG, "no candidate geometry for L=%d", in->L);
    float best = -1.f, best_score = 0.f;
    for (const elp_job_spec& c : cand) {
        std::vector<elp_job_spec> specs((size_t)copies, c);
        for (int k = 0; k < copies; k++) specs[(size_t)k].seed = c.seed + (uint32_t)k;
        elp_batch* b = nullptr;
        if (elp_batch_create(specs.data(), copies, in->device, &b) != ELP_OK) continue;
        float ms = 0.f;
        elp_status st = elp_batch_init_melts(b);
        if (st == ELP_OK) st = elp_batch_run(b, steps);  // warm-up (and graph capture)
        if (st == ELP_OK) st = elp_batch_run_timed(b, steps, &ms);
        elp_batch_destroy(b);
        if (st != ELP_OK) continue;
        // Tile walls slow the melt's clock: a tiled step moves the rings as
        // far as f efpol steps (f measured per shape, 1 for the wall-free
        // whole box), so candidates compete on time per efpol-equivalent step.
        const float per = ms / (float)steps;
        const float score = per / (float)clock_factor(c);
        if (best < 0.f || score < best_score) {
            best = per;
            best_score = score;
            *out = c;
        }
    }
    if (best < 0.f) return elp_fail(ELP_ERR_CUDA, "no candidate geometry could be run");
    // make the choice explicit
    int P;
    elp_geometry g;
    elp_resolve_spec(out, &P, &g);
    out->periodic = g.periodic;
    out->tile[0] = g.tx; out->tile[1] = g.ty; out->tile[2] = g.tz;
    out->ncol = g.ncol;
    if (ms_per_step) *ms_per_step = best;
    return ELP_OK;
}
