// elp_api.cu -- the single-melt C ABI (include/elp.h): one melt on one GPU,
// run as a group of one (elp_group.h) so that it executes exactly the kernel
// path a batch uses.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include "elp_common.h"
#include "elp_group.h"
#include "elp_kernels.h"

struct elp_ctx {
    elp_geometry g;
    int N = 0, P = 0;
    int linear = 0;
    uint32_t seed = 0, salt = 0;
    int device = 0;
    int nsm = 148;
    int domains = 0, threads = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t* d_lat = nullptr;
    uint32_t* d_rec = nullptr;
    uint32_t* d_table = nullptr;
    unsigned long long* d_acc = nullptr;  // [0] accepted moves, [1] device error flags
    size_t device_bytes = 0;
    int loaded = 0;
    elp_group G;
    int group_ready = 0;
    elp_walk_bufs wb;
};

static uint32_t* error_flags(elp_ctx* c) { return reinterpret_cast<uint32_t*>(c->d_acc + 1); }

extern "C" elp_status elp_create(const elp_job_spec* spec, elp_ctx** out)
{
    if (!spec || !out) return elp_fail(ELP_ERR_ARG, "null argument");
    *out = nullptr;
    int P = 0;
    elp_geometry g;
    elp_status st = elp_resolve_spec(spec, &P, &g);
    if (st) return st;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return elp_fail(ELP_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (spec->device < 0 || spec->device >= ndev) return elp_fail(ELP_ERR_ARG, "device %d not present", spec->device);
    ELP_CUDA_TRY(cudaSetDevice(spec->device));

    elp_ctx* c = new (std::nothrow) elp_ctx();
    if (!c) return elp_fail(ELP_ERR_NOMEM, "host allocation failed");
    c->g = g;
    c->N = spec->N;
    c->P = P;
    c->linear = spec->linear;
    c->seed = spec->seed;
    c->salt = spec->salt;
    c->device = spec->device;
    if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, spec->device) != cudaSuccess || c->nsm < 1)
        c->nsm = 148;
    elp_smem_layout lay;
    elp_layout(&g, &lay);
    c->domains = g.periodic ? 1 : (g.L / g.tx) * (g.L / g.ty) * (g.L / g.tz);
    c->threads = (lay.groups + 31) / 32 * 32;

    const size_t S = (size_t)g.L * g.L * g.L;
#define ALLOC(ptr, bytes)                                                                                  \
    do {                                                                                                   \
        cudaError_t ea_ = cudaMalloc((void**)&(ptr), (bytes));                                             \
        if (ea_ != cudaSuccess) {                                                                          \
            st = elp_fail(ELP_ERR_NOMEM, "cudaMalloc(%zu): %s", (size_t)(bytes), cudaGetErrorString(ea_)); \
            goto bad;                                                                                      \
        }                                                                                                  \
        c->device_bytes += (bytes);                                                                        \
    } while (0)
    ALLOC(c->d_lat, S * sizeof(uint32_t));
    ALLOC(c->d_rec, (size_t)P * ELP_REC_WORDS * sizeof(uint32_t));
    ALLOC(c->d_table, 4096);
    ALLOC(c->d_acc, 8 * sizeof(unsigned long long));
#undef ALLOC
    {
        uint8_t tab[4096];
        elp_build_table(tab);
        if (cudaMemcpy(c->d_table, tab, 4096, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(c->d_lat, 0, S * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemset(c->d_acc, 0, 8 * sizeof(unsigned long long)) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
            st = elp_fail(ELP_ERR_CUDA, "context set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
            goto bad;
        }
        cudaError_t eg = elp_group_init(&c->G, g, c->nsm, spec->kernel == 1, spec->steps_per_launch, c->d_table,
                                        error_flags(c), c->stream);
        if (eg == cudaSuccess) {
            c->group_ready = 1;
            elp_group_add(&c->G, c->d_lat, c->d_rec, c->d_acc, c->N, c->P, c->seed, c->salt, 0, c->linear);
            eg = elp_group_commit(&c->G);
        }
        if (eg != cudaSuccess) {
            st = elp_fail(ELP_ERR_CUDA, "group set-up failed: %s", cudaGetErrorString(eg));
            goto bad;
        }
        if (c->linear && !c->G.specialised) {
            st = elp_fail(ELP_ERR_ARG, "linear chains need a domain shape with a specialised kernel (L=%d tile %dx%dx%d)",
                          g.L, g.tx, g.ty, g.tz);
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
    if (c->group_ready) elp_group_free(&c->G);
    elp_walk_bufs_free(&c->wb);
    cudaFree(c->d_lat); cudaFree(c->d_rec); cudaFree(c->d_table); cudaFree(c->d_acc);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static elp_status upload(elp_ctx* c, const uint32_t* lat, const uint32_t* rec, uint64_t step)
{
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    ELP_CUDA_TRY(cudaMemcpyAsync(c->d_lat, lat, S * 4, cudaMemcpyHostToDevice, c->stream));
    ELP_CUDA_TRY(cudaMemcpyAsync(c->d_rec, rec, (size_t)c->P * ELP_REC_WORDS * 4, cudaMemcpyHostToDevice, c->stream));
    ELP_CUDA_TRY(elp_group_set_step(&c->G, 0, step));
    // a new configuration replaces whatever an earlier failed launch left
    ELP_CUDA_TRY(cudaMemsetAsync(error_flags(c), 0, sizeof(uint32_t), c->stream));
    ELP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->loaded = 1;
    return ELP_OK;
}

extern "C" elp_status elp_load_chains(elp_ctx* c, const int32_t* start, const uint8_t* bonds, uint64_t step)
{
    if (!c || !start || !bonds) return elp_fail(ELP_ERR_ARG, "null argument");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    // the lattice is rebuilt in place on the device: until that succeeds the
    // context holds no configuration.  The step is queued ahead of the build,
    // whose status read-back is the call's one synchronisation.
    c->loaded = 0;
    ELP_CUDA_TRY(elp_group_set_step(&c->G, 0, step));
    ELP_CUDA_TRY(cudaMemsetAsync(error_flags(c), 0, sizeof(uint32_t), c->stream));
    elp_status st = elp_build_melt(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, start, bonds, &c->wb, c->stream);
    if (st) return st;
    c->loaded = 1;
    return ELP_OK;
}

extern "C" elp_status elp_init_melt(elp_ctx* c)
{
    if (!c) return elp_fail(ELP_ERR_ARG, "null context");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    c->loaded = 0;
    elp_status st = elp_init_melt_device(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, c->stream);
    if (st) return st;
    ELP_CUDA_TRY(elp_group_set_step(&c->G, 0, 0));
    ELP_CUDA_TRY(cudaMemsetAsync(error_flags(c), 0, sizeof(uint32_t), c->stream));
    ELP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->loaded = 1;
    return ELP_OK;
}

extern "C" elp_status elp_set_state(elp_ctx* c, const uint32_t* words, const uint32_t* records, uint64_t step)
{
    if (!c || !words || !records) return elp_fail(ELP_ERR_ARG, "null argument");
    return upload(c, words, records, step);
}

extern "C" elp_status elp_get_state(elp_ctx* c, uint32_t* words, uint32_t* records)
{
    if (!c || !words || !records) return elp_fail(ELP_ERR_ARG, "null argument");
    size_t S = (size_t)c->g.L * c->g.L * c->g.L;
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    ELP_CUDA_TRY(cudaMemcpyAsync(words, c->d_lat, S * 4, cudaMemcpyDeviceToHost, c->stream));
    ELP_CUDA_TRY(cudaMemcpyAsync(records, c->d_rec, (size_t)c->P * ELP_REC_WORDS * 4, cudaMemcpyDeviceToHost, c->stream));
    return elp_device_errors(error_flags(c), c->stream);
}

extern "C" elp_status elp_run(elp_ctx* c, int64_t nsteps)
{
    if (!c) return elp_fail(ELP_ERR_ARG, "null context");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    if (nsteps < 0) return elp_fail(ELP_ERR_ARG, "negative step count");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    ELP_CUDA_TRY(elp_group_run(&c->G, nsteps));
    return ELP_OK;
}

extern "C" elp_status elp_run_timed(elp_ctx* c, int64_t nsteps, float* ms)
{
    if (!c || !ms) return elp_fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    if (nsteps < 0) return elp_fail(ELP_ERR_ARG, "negative step count");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    // work already queued on the stream (a cache flush, copies) runs before
    // ev0 is reached, so the events bracket only these launches
    ELP_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
    ELP_CUDA_TRY(elp_group_run(&c->G, nsteps));
    ELP_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
    ELP_CUDA_TRY(cudaEventSynchronize(c->ev1));
    ELP_CUDA_TRY(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return elp_device_errors(error_flags(c), c->stream);
}

extern "C" void* elp_stream(elp_ctx* c)
{
    return c ? static_cast<void*>(c->stream) : nullptr;
}

extern "C" elp_status elp_sync(elp_ctx* c)
{
    if (!c) return elp_fail(ELP_ERR_ARG, "null context");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    return elp_device_errors(error_flags(c), c->stream);
}

extern "C" elp_status elp_accepted(elp_ctx* c, uint64_t* acc)
{
    if (!c || !acc) return elp_fail(ELP_ERR_ARG, "null argument");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    unsigned long long v = 0;
    ELP_CUDA_TRY(cudaMemcpyAsync(&v, c->d_acc, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    ELP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    *acc = v;
    return elp_device_errors(error_flags(c), c->stream);
}

extern "C" elp_status elp_debug_waits(elp_ctx* c, uint32_t polls, int32_t hold_block)
{
    if (!c) return elp_fail(ELP_ERR_ARG, "null context");
    if (hold_block < -1 || (c->G.nitems > 0 && hold_block >= c->G.nitems))
        return elp_fail(ELP_ERR_ARG, "block %d not in 0..%d", hold_block, c->G.nitems - 1);
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    ELP_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->G.wait_polls = polls;
    c->G.hold_cta1 = hold_block + 1;
    if (c->G.graph) {
        // captured launches carry the old bound: capture again on the next run
        cudaGraphExecDestroy(c->G.graph);
        c->G.graph = nullptr;
    }
    return ELP_OK;
}

extern "C" elp_status elp_fetch_chains(elp_ctx* c, int32_t* start, uint8_t* bonds)
{
    if (!c || !start || !bonds) return elp_fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    // the walk is queued straight behind the steps (no host round trip in
    // between); the launches' error flags are read after it and take
    // precedence over the walk's status
    elp_status st = elp_fetch_rings(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, &c->wb, start, bonds, c->stream);
    elp_status fl = elp_device_errors(error_flags(c), c->stream);
    return fl ? fl : st;
}

extern "C" elp_status elp_fetch_checked(elp_ctx* c, int32_t* start, uint8_t* bonds, int32_t* code)
{
    if (!c || !start || !bonds || !code) return elp_fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    elp_status st = elp_fetch_checked_melt(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, &c->wb, start, bonds,
                                           code, c->stream);
    elp_status fl = elp_device_errors(error_flags(c), c->stream);
    return fl ? fl : st;
}

extern "C" elp_status elp_observe(elp_ctx* c, double* cms_tuv, double* rg2, double* sl, uint64_t* run_hist,
                                  int32_t nbins)
{
    if (!c) return elp_fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    elp_status st = elp_device_errors(error_flags(c), c->stream);
    if (st) return st;
    return elp_observe_melt(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, &c->wb, cms_tuv, rg2, sl, run_hist, nbins,
                            c->stream);
}

extern "C" elp_status elp_check(elp_ctx* c, int32_t* code)
{
    if (!c || !code) return elp_fail(ELP_ERR_ARG, "null argument");
    if (!c->loaded) return elp_fail(ELP_ERR_STATE, "no configuration loaded");
    ELP_CUDA_TRY(cudaSetDevice(c->device));
    elp_status st = elp_device_errors(error_flags(c), c->stream);
    if (st) return st;
    return elp_check_melt(c->d_lat, c->d_rec, c->g.L, c->N, c->P, c->linear, &c->wb, code, c->stream);
}

extern "C" elp_status elp_get_info(const elp_ctx* c, elp_info* info)
{
    if (!c || !info) return elp_fail(ELP_ERR_ARG, "null argument");
    memset(info, 0, sizeof(*info));
    info->L = c->g.L; info->N = c->N; info->P = c->P;
    info->periodic = c->g.periodic;
    info->tile[0] = c->g.tx; info->tile[1] = c->g.ty; info->tile[2] = c->g.tz;
    info->ncol = c->g.ncol;
    info->domains = c->domains;
    info->threads = c->G.threads;
    info->specialised = c->G.specialised;
    info->smem_bytes = c->G.smem;
    info->step = elp_group_step(&c->G, 0);
    info->device_bytes = c->device_bytes + c->wb.bytes;
    info->linear = c->linear;
    info->kernels = c->G.kernels;
    return ELP_OK;
}

extern "C" elp_status elp_write_tuv(elp_ctx* c, const char* path)
{
    if (!c || !path) return elp_fail(ELP_ERR_ARG, "null argument");
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
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", path);
    size_t wr = fwrite(text.data(), 1, len, f);
    int cl = fclose(f);
    if (wr != len || cl) return elp_fail(ELP_ERR_IO, "short write to %s", path);
    return ELP_OK;
}

extern "C" elp_status elp_load_tuv(elp_ctx* c, const char* path, uint64_t step)
{
    if (!c || !path) return elp_fail(ELP_ERR_ARG, "null argument");
    char* text = nullptr;
    size_t len = 0;
    elp_status st = elp_read_file(path, &text, &len);
    if (st) return st;
    std::vector<int32_t> start((size_t)c->P * 3);
    std::vector<uint8_t> bonds((size_t)c->P * c->N);
    st = elp_parse_tuv(text, path, c->g.L, c->N, c->P, start.data(), bonds.data());
    free(text);
    if (st) return st;
    return elp_load_chains(c, start.data(), bonds.data(), step);
}
