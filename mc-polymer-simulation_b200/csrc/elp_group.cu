// elp_group.cu -- launching the sweep for a group of melts (see elp_group.h).
#include <string.h>

#include "elp_group.h"

namespace {
__global__ void ctr_add_kernel(uint32_t* c, uint32_t v) { *c += v; }

int domains_of(const elp_geometry& g)
{
    return g.periodic ? 1 : (g.L / g.tx) * (g.L / g.ty) * (g.L / g.tz);
}

Sweep2Launch make_launch(const elp_group* G, int nsteps, uint32_t step_base, int check_only)
{
    Sweep2Launch l;
    memset(&l, 0, sizeof(l));
    l.geom = G->g;
    l.sx = G->lay.sx;
    l.sxy = G->lay.sxy;
    l.nsm = G->nsm;
    l.check_only = check_only;
    double sites = (double)G->g.tx * G->g.ty * G->g.tz, box = (double)G->g.L * G->g.L * G->g.L;
    for (const BatchJob& j : G->jobs) {
        double m = j.nchains * sites / box;
        if (m > l.max_runs_per_domain) l.max_runs_per_domain = m;
        if (j.linear) l.linear = 1;
    }
    l.args.jobs = G->d_jobs;
    l.args.items = G->d_items;
    l.args.nitems = G->nitems;
    l.args.nsteps = nsteps;
    l.args.step_base = step_base;
    l.args.step_dev = G->d_ctr;
    l.args.table = G->d_table;
    l.args.error = G->d_error;
    l.args.grid_bar = G->d_ctr + 1;
    l.args.wait_polls = G->wait_polls;
    l.args.hold_cta1 = G->hold_cta1;
    return l;
}

// Generic kernel: one launch per melt, absolute step known on the host.
cudaError_t launch_generic(elp_group* G, int nsteps)
{
    for (size_t j = 0; j < G->jobs.size(); j++) {
        const BatchJob& J = G->jobs[j];
        SweepArgs a;
        memset(&a, 0, sizeof(a));
        a.lat = J.lat;
        a.rec = J.rec;
        a.table = G->d_table;
        a.accepted = J.acc;
        a.error = G->d_error;
        a.nchains = J.nchains;
        a.L = G->g.L;
        a.periodic = G->g.periodic;
        a.tx = G->g.tx; a.ty = G->g.ty; a.tz = G->g.tz;
        a.ncol = G->g.ncol;
        a.sx = G->lay.sx; a.sxy = G->lay.sxy; a.ox = G->lay.ox;
        a.words = G->lay.words;
        a.groups = G->lay.groups;
        a.seed = J.seed;
        a.salt = J.salt;
        a.step0 = (uint32_t)(J.step0 + (uint32_t)G->steps_done);
        a.nsteps = nsteps;
        int threads = (G->lay.groups + 31) / 32 * 32;
        cudaError_t e = elp_launch_sweep(&a, domains_of(G->g), threads < 32 ? 32 : threads, G->lay.bytes, G->stream);
        if (e != cudaSuccess) return e;
        G->kernels++;
    }
    return cudaSuccess;
}

cudaError_t launch_once(elp_group* G, int nsteps, uint32_t step_base)
{
    if (!G->specialised) return launch_generic(G, nsteps);
    Sweep2Launch l = make_launch(G, nsteps, step_base, 0);
    G->kernels++;
    return elp_launch_sweep2(&l, G->stream);
}
}  // namespace

cudaError_t elp_group_init(elp_group* G, const elp_geometry& geom, int nsm, int generic, int spl,
                           const uint32_t* d_table, uint32_t* d_error, cudaStream_t stream)
{
    G->g = geom;
    elp_layout(&geom, &G->lay);
    G->nsm = nsm;
    G->generic = generic;
    G->spl = spl > 0 ? spl : 1;
    G->use_graph = !geom.periodic;
    G->graph_steps = 100;
    G->stream = stream;
    G->d_table = d_table;
    G->d_error = d_error;
    // step counter and the two counts of the grid barrier of tiled launches,
    // stream-ordered (a group created while others run does not stall them)
    cudaError_t e = cudaMallocAsync((void**)&G->d_ctr, 4 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(G->d_ctr, 0, 4 * sizeof(uint32_t), stream);
}

void elp_group_add(elp_group* G, uint32_t* lat, uint32_t* rec, unsigned long long* acc, int N, int nchains,
                   uint32_t seed, uint32_t salt, uint64_t step, int linear)
{
    BatchJob j;
    memset(&j, 0, sizeof(j));
    j.linear = linear;
    j.lat = lat;
    j.rec = rec;
    j.acc = acc;
    j.L = G->g.L;
    j.nchains = nchains;
    j.ntx = G->g.periodic ? 1 : G->g.L / G->g.tx;
    j.nty = G->g.periodic ? 1 : G->g.L / G->g.ty;
    j.ntz = G->g.periodic ? 1 : G->g.L / G->g.tz;
    j.seed = seed;
    j.salt = salt;
    j.step0 = (uint32_t)(step - G->steps_done);
    G->jobs.push_back(j);
    G->N.push_back(N);
}

cudaError_t elp_group_commit(elp_group* G)
{
    const int nd = domains_of(G->g);
    const size_t nj = G->jobs.size();
    cudaError_t e;
    // the tables grow only, stream-ordered: a membership change (the serving
    // loop commits every few ticks) synchronises nothing but this group
    if (nj > G->cap_jobs) {
        if (G->d_jobs && (e = cudaFreeAsync(G->d_jobs, G->stream)) != cudaSuccess) return e;
        G->d_jobs = nullptr;
        G->cap_jobs = 0;
        const size_t cap = nj < 16 ? 16 : 2 * nj;
        if ((e = cudaMallocAsync((void**)&G->d_jobs, cap * sizeof(BatchJob), G->stream)) != cudaSuccess) return e;
        G->cap_jobs = cap;
    }
    if (nj * nd > G->cap_items) {
        if (G->d_items && (e = cudaFreeAsync(G->d_items, G->stream)) != cudaSuccess) return e;
        G->d_items = nullptr;
        G->cap_items = 0;
        const size_t cap = nj * nd < 64 ? 64 : 2 * nj * nd;
        if ((e = cudaMallocAsync((void**)&G->d_items, cap * sizeof(uint2), G->stream)) != cudaSuccess) return e;
        G->cap_items = cap;
    }
    std::vector<uint2> items(nj * nd);
    // domain-major order: the first wave of a persistent grid spreads over melts
    for (int d = 0; d < nd; d++)
        for (size_t j = 0; j < nj; j++) items[(size_t)d * nj + j] = make_uint2((uint32_t)j, (uint32_t)d);
    G->nitems = (int)items.size();
    if ((e = cudaMemcpyAsync(G->d_jobs, G->jobs.data(), nj * sizeof(BatchJob), cudaMemcpyHostToDevice, G->stream)))
        return e;
    if ((e = cudaMemcpyAsync(G->d_items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                             G->stream)))
        return e;
    Sweep2Launch l = make_launch(G, G->g.periodic ? G->spl : 1, 0, 1);
    G->specialised = !G->generic && elp_launch_sweep2(&l, G->stream) == cudaSuccess;
    if (G->specialised) {
        G->threads = l.threads_out;
        G->smem = l.smem_out;
    } else {
        G->threads = (G->lay.groups + 31) / 32 * 32;
        G->threads = G->threads < 32 ? 32 : G->threads;
        G->smem = G->lay.bytes;
    }
    if (G->graph) {
        cudaGraphExecDestroy(G->graph);
        G->graph = nullptr;
    }
    return cudaStreamSynchronize(G->stream);
}

cudaError_t elp_group_set_step(elp_group* G, int j, uint64_t step)
{
    G->jobs[(size_t)j].step0 = (uint32_t)(step - G->steps_done);
    return cudaMemcpyAsync(G->d_jobs + j, &G->jobs[(size_t)j], sizeof(BatchJob), cudaMemcpyHostToDevice, G->stream);
}

uint64_t elp_group_step(const elp_group* G, int j)
{
    return (uint64_t)G->jobs[(size_t)j].step0 + G->steps_done;
}

cudaError_t elp_group_run(elp_group* G, int64_t nsteps)
{
    cudaError_t e;
    if (G->g.periodic) {
        while (nsteps > 0) {
            int k = (int)(nsteps < G->spl ? nsteps : G->spl);
            if ((e = launch_once(G, k, (uint32_t)(G->steps_done - G->ctr_mirror))) != cudaSuccess) return e;
            G->steps_done += (uint64_t)k;
            nsteps -= k;
        }
        return cudaSuccess;
    }
    // tiled domains: the specialised kernel takes spl steps per (cooperative)
    // launch, the generic one a single step
    const int k = G->specialised ? G->spl : 1;
    const int gsteps = G->graph_steps > k ? G->graph_steps / k * k : k;
    if (G->specialised && G->use_graph && nsteps >= gsteps) {
        const uint32_t base = (uint32_t)(G->steps_done - G->ctr_mirror);
        if (!G->graph || G->graph_base != base) {
            if (G->graph) cudaGraphExecDestroy(G->graph);
            G->graph = nullptr;
            cudaGraph_t gr;
            if ((e = cudaStreamBeginCapture(G->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
            for (int i = 0; i < gsteps; i += k) {
                Sweep2Launch l = make_launch(G, k, base + (uint32_t)i, 0);
                elp_launch_sweep2(&l, G->stream);
            }
            ctr_add_kernel<<<1, 1, 0, G->stream>>>(G->d_ctr, (uint32_t)gsteps);
            if ((e = cudaStreamEndCapture(G->stream, &gr)) != cudaSuccess) return e;
            e = cudaGraphInstantiate(&G->graph, gr, 0);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) return e;
            G->graph_base = base;
        }
        while (nsteps >= gsteps) {
            if ((e = cudaGraphLaunch(G->graph, G->stream)) != cudaSuccess) return e;
            G->kernels += (uint64_t)(gsteps / k + 1);   // its sweep launches and the counter update
            G->steps_done += (uint64_t)gsteps;
            G->ctr_mirror += (uint32_t)gsteps;
            nsteps -= gsteps;
        }
    }
    while (nsteps > 0) {
        const int kk = (int)(nsteps < k ? nsteps : k);
        if ((e = launch_once(G, kk, (uint32_t)(G->steps_done - G->ctr_mirror))) != cudaSuccess) return e;
        G->steps_done += (uint64_t)kk;
        nsteps -= kk;
    }
    return cudaSuccess;
}

void elp_group_free(elp_group* G)
{
    if (G->graph) cudaGraphExecDestroy(G->graph);
    if (G->stream) cudaStreamSynchronize(G->stream);
    cudaFree(G->d_jobs);
    cudaFree(G->d_items);
    cudaFree(G->d_ctr);
    G->graph = nullptr;
    G->d_jobs = nullptr;
    G->d_items = nullptr;
    G->d_ctr = nullptr;
}
