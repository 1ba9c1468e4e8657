// elp_server.cu -- the serving loop: continuous batching of melt jobs.
//
// Jobs (a melt spec, a step count, a dump interval) arrive at any time.  Each
// domain geometry has a group (elp_group.h) with its own stream, and every
// group ticks on its own: a tick is `quantum` steps of all its members, and
// when a group's tick ends the scheduler thread does its bookkeeping, admits
// queued jobs whose device memory fits the HBM budget, retires finished ones
// and launches its next tick at once -- no group waits for another, so a
// small latency-bound melt never holds up the GPU.  Lattices stay resident
// between dumps.  At a dump the job's state is copied device-to-device on
// the group's stream at the end of the tick; I/O threads, each with its own
// stream, scratch and pinned host buffers, rebuild the rings from the copy,
// check the melt's invariants (every dump, as CheckIntegrity), and format
// and write the TUV text while the group keeps computing.  A dump that fails
// its check or its write ends the job with that status at the group's next
// tick.  Queued jobs are admitted in order; a job that does not fit the
// budget lets smaller ones behind it pass, until it has been passed
// ADMIT_PASSES times: then it holds its place and the memory it waits for.  A job follows
// the same trajectory alone, in any mix, or through the single-melt API: its
// kernel, counters and geometry depend only on its spec.
//
// The reference runs one fixed job per process (gpupol2/gpupol2.c:14-70 with
// a synchronous dump per interval, gpupol2/gpupol_cuda.cu:52-76); it has no
// serving mode.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "elp_common.h"
#include "elp_group.h"
#include "elp_kernels.h"

namespace {

uint64_t fnv1a(uint64_t h, const void* p, size_t n)
{
    const uint8_t* b = (const uint8_t*)p;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}

struct SJob {
    uint64_t id = 0;
    elp_job_spec spec;
    elp_geometry g;
    int P = 0;
    int64_t nsteps = 0, dump_interval = 0, done_steps = 0;
    std::string dir;
    double t_submit = 0, t_start = 0, t_done = 0;
    uint32_t dumps = 0;
    size_t bytes = 0;
    uint32_t* lat = nullptr;
    uint32_t* rec = nullptr;
    int group = -1, index = -1;
    elp_status status = ELP_OK;
    int integrity = -1;
    uint64_t checksum = 0;
    std::string error;
    int passed = 0;                       // queued: times a job behind it was admitted first
    std::atomic<int> abort{0};            // set by an I/O thread: a dump failed (status code)
    std::atomic<int> pending{0};          // snapshots queued or in work
    std::atomic<bool> final_seen{false};  // the last snapshot (or the abort marker) is done
};

// A snapshot on its way to the host.  An abort marker (no state) ends a job
// whose dump failed.
struct Snap {
    SJob* job = nullptr;
    int64_t step = 0;
    bool final = false;
    bool abort = false;
    uint32_t* d_lat = nullptr;            // copy of the job's state at `step`
    uint32_t* d_rec = nullptr;
    cudaEvent_t ready = nullptr;          // recorded after the copy on the group's stream
};

struct SGroup {
    std::tuple<int, int, int, int, int, int, int> key;   // geometry, linear chains
    elp_group G;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;             // end of the running tick
    std::vector<SJob*> members;           // resident jobs, including ones admitted during a tick
    std::vector<SJob*> running;           // the members of the running tick
    bool dirty = false;                   // members changed since the job table was built
    bool busy = false;                    // a tick is in flight
};

}  // namespace

struct elp_server {
    elp_server_opts o;
    int nsm = 148;
    std::chrono::steady_clock::time_point t0;
    uint32_t* d_table = nullptr;
    uint32_t* d_err = nullptr;            // 64 groups x 4 words
    uint32_t* h_err = nullptr;            // pinned: word 0 of each group's flags, copied at the end of its tick
    unsigned long long* d_acc = nullptr;  // accepted moves (all jobs together)

    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<SJob*> queue;
    std::vector<SJob*> finished;          // results not yet polled
    uint64_t next_id = 1;
    std::atomic<bool> stop{false};
    std::atomic<bool> io_stop{false};     // set after the scheduler has finished
    uint64_t submitted = 0, completed = 0;
    size_t bytes_in_use = 0;
    double moves_done = 0;
    elp_status fatal = ELP_OK;
    std::string fatal_msg;

    std::vector<std::unique_ptr<SGroup>> groups;
    std::vector<SJob*> resident;

    std::mutex io_mu;
    std::condition_variable io_cv;
    std::deque<Snap> io_q;
    std::vector<std::thread> io_threads;
    std::atomic<int> io_busy{0};
    std::thread sched;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

static void fail_job(elp_server* s, SJob* j, elp_status st, const char* msg);

// Publish a finished job once its last snapshot and every earlier one are
// done (several I/O threads may hold snapshots of one job).
static void snapshot_done(elp_server* s, SJob* j, bool last)
{
    if (last) j->final_seen = true;
    if (--j->pending == 0 && j->final_seen.load()) {
        std::lock_guard<std::mutex> lk(s->mu);
        j->t_done = s->now();
        s->finished.push_back(j);
        s->completed++;
        s->cv_done.notify_all();
    }
}

// A dump failed: the first failure decides the job's status.
static void dump_failed(elp_server* s, SJob* j, elp_status st, const std::string& msg)
{
    int expect = 0;
    if (j->abort.compare_exchange_strong(expect, (int)st)) {
        std::lock_guard<std::mutex> lk(s->mu);
        j->status = st;
        j->error = msg;
    }
}

// Write a TUV file; ELP_ERR_IO on any failure (open, short write, close).
static elp_status write_text(const char* path, const std::string& text, size_t len)
{
    FILE* f = fopen(path, "wb");
    if (!f) return elp_fail(ELP_ERR_IO, "cannot open %s for writing", path);
    const size_t n = fwrite(text.data(), 1, len, f);
    const int c = fclose(f);
    if (n != len || c != 0) return elp_fail(ELP_ERR_IO, "writing %s failed (%zu of %zu bytes)", path, n, len);
    return ELP_OK;
}

// One I/O thread: rebuilds the rings of snapshots on its own stream and
// scratch into pinned host buffers, checks the melt's invariants, writes its
// TUV text.
static void io_worker(elp_server* s)
{
    cudaSetDevice(s->o.device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    elp_walk_bufs wb;
    int32_t* h_start = nullptr;   // pinned, grown as jobs need
    uint8_t* h_bonds = nullptr;
    size_t cap_start = 0, cap_bonds = 0;
    for (;;) {
        Snap sn;
        {
            std::unique_lock<std::mutex> lk(s->io_mu);
            s->io_cv.wait(lk, [&] { return s->io_stop.load() || !s->io_q.empty(); });
            if (s->io_q.empty()) break;
            sn = s->io_q.front();
            s->io_q.pop_front();
        }
        SJob* j = sn.job;
        if (sn.abort) {
            snapshot_done(s, j, true);
            s->io_busy--;
            continue;
        }
        const int L = j->g.L, N = j->spec.N, P = j->P;
        elp_status rc = ELP_OK;
        if ((size_t)P * 3 > cap_start) {
            cudaFreeHost(h_start);
            h_start = nullptr;
            cap_start = 0;
            if (cudaMallocHost((void**)&h_start, (size_t)P * 3 * sizeof(int32_t)) == cudaSuccess)
                cap_start = (size_t)P * 3;
            else
                rc = elp_fail(ELP_ERR_NOMEM, "pinned host buffer of %d rings", P);
        }
        if (rc == ELP_OK && (size_t)P * N > cap_bonds) {
            cudaFreeHost(h_bonds);
            h_bonds = nullptr;
            cap_bonds = 0;
            if (cudaMallocHost((void**)&h_bonds, (size_t)P * N) == cudaSuccess)
                cap_bonds = (size_t)P * N;
            else
                rc = elp_fail(ELP_ERR_NOMEM, "pinned host buffer of %d x %d bonds", P, N);
        }
        cudaStreamWaitEvent(st, sn.ready, 0);
        const int lin = j->spec.linear ? 1 : 0;
        int32_t code = -1;
        if (rc == ELP_OK)
            rc = elp_fetch_checked_melt(sn.d_lat, sn.d_rec, L, N, P, lin, &wb, h_start, h_bonds, &code, st);
        std::string err = rc == ELP_OK ? std::string() : std::string(elp_last_error());
        cudaFreeAsync(sn.d_lat, st);
        cudaFreeAsync(sn.d_rec, st);
        cudaStreamSynchronize(st);
        cudaEventDestroy(sn.ready);
        if (rc == ELP_OK) {
            if (sn.final || code != 0) {
                std::lock_guard<std::mutex> lk(s->mu);
                j->integrity = code;
            }
            if (code != 0) {
                rc = ELP_ERR_INTEGRITY;
                char m[160];
                snprintf(m, sizeof(m), "integrity check failed at step %lld (code %d)", (long long)sn.step, code);
                err = m;
            }
        }
        if (rc == ELP_OK && !j->dir.empty()) {
            size_t len = 0;
            elp_format_tuv(L, N, P, h_start, h_bonds, nullptr, 0, &len);
            std::string text(len + 1, '\0');
            elp_format_tuv(L, N, P, h_start, h_bonds, &text[0], len + 1, &len);
            char path[4096];
            snprintf(path, sizeof(path), "%s/t=%lld_dev=0.res", j->dir.c_str(), (long long)sn.step);
            rc = write_text(path, text, len);
            if (rc != ELP_OK) err = elp_last_error();
        }
        if (rc != ELP_OK) {
            dump_failed(s, j, rc, err);
        } else if (sn.final) {
            uint64_t h = 0xcbf29ce484222325ULL;
            h = fnv1a(h, h_start, (size_t)P * 3 * sizeof(int32_t));
            h = fnv1a(h, h_bonds, (size_t)P * N);
            j->checksum = h;
        }
        snapshot_done(s, j, sn.final);
        s->io_busy--;
    }
    elp_walk_bufs_free(&wb);
    cudaFreeHost(h_start);
    cudaFreeHost(h_bonds);
    cudaStreamDestroy(st);
}

static SGroup* group_for(elp_server* s, SJob* j)
{
    auto key = std::make_tuple(j->g.periodic, j->g.L, j->g.tx, j->g.ty, j->g.tz, j->g.ncol, j->spec.linear ? 1 : 0);
    for (auto& gp : s->groups)
        if (gp->key == key) return gp.get();
    if (s->groups.size() >= 64) return nullptr;
    std::unique_ptr<SGroup> gp(new SGroup());
    gp->key = key;
    if (cudaStreamCreateWithFlags(&gp->s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    if (cudaEventCreateWithFlags(&gp->ev, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    if (elp_group_init(&gp->G, j->g, s->nsm, 0, s->o.quantum, s->d_table, s->d_err + 4 * s->groups.size(), gp->s) !=
        cudaSuccess)
        return nullptr;
    // membership changes every few ticks: a captured graph would be rebuilt
    // about as often as it is replayed, so tiled groups launch directly, one
    // step per launch (a launch of several tiled steps is cooperative and
    // holds every SM it uses until its last step, stalling the other groups)
    gp->G.use_graph = 0;
    if (!j->g.periodic) gp->G.spl = 1;
    s->groups.push_back(std::move(gp));
    return s->groups.back().get();
}

static void fail_job(elp_server* s, SJob* j, elp_status st, const char* msg)
{
    j->status = st;
    j->error = msg;
    std::lock_guard<std::mutex> lk(s->mu);
    j->t_done = s->now();
    s->finished.push_back(j);
    s->completed++;
    s->cv_done.notify_all();
}

// Admit queued jobs that fit the budget; returns false on a fatal CUDA error.
// Jobs are taken in queue order.  A job that does not fit the memory left
// lets the jobs behind it pass (no head-of-line blocking) until it has been
// passed ADMIT_PASSES times; from then on it sets aside the memory it needs,
// and a job behind it is admitted only if it fits next to everything set
// aside ahead of it, so a large job is never starved by a stream of small
// ones.  The scan looks at most ADMIT_SCAN queued jobs.
static constexpr int ADMIT_SCAN = 256;
static constexpr int ADMIT_PASSES = 64;
static bool admit(elp_server* s)
{
    std::vector<SJob*> take, refuse;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        size_t in_use = s->bytes_in_use, reserved = 0;
        const size_t budget = s->o.hbm_budget;
        std::vector<SJob*> waiting;           // jobs ahead that did not fit
        int scanned = 0;
        for (auto it = s->queue.begin(); it != s->queue.end() && scanned < ADMIT_SCAN; scanned++) {
            if (s->resident.size() + take.size() >= (size_t)s->o.max_jobs) break;
            SJob* c = *it;
            if (c->bytes > budget) {
                refuse.push_back(c);
                it = s->queue.erase(it);
            } else if (in_use + reserved + c->bytes <= budget) {
                take.push_back(c);
                in_use += c->bytes;
                for (SJob* w : waiting) w->passed++;
                it = s->queue.erase(it);
            } else {
                waiting.push_back(c);
                if (c->passed >= ADMIT_PASSES) reserved += c->bytes;
                if (in_use + reserved >= budget) break;   // nothing behind it can pass
                ++it;
            }
        }
    }
    for (SJob* j : refuse) fail_job(s, j, ELP_ERR_BUSY, "job needs more device memory than the server budget");
    for (SJob* j : take) {
        SGroup* gp = group_for(s, j);
        if (!gp) {
            fail_job(s, j, ELP_ERR_CUDA, "cannot create a group for the job");
            continue;
        }
        const size_t S = (size_t)j->g.L * j->g.L * j->g.L;
        if (cudaMallocAsync((void**)&j->lat, S * 4, gp->s) != cudaSuccess ||
            cudaMallocAsync((void**)&j->rec, (size_t)j->P * ELP_REC_WORDS * 4, gp->s) != cudaSuccess) {
            fail_job(s, j, ELP_ERR_NOMEM, "device allocation failed");
            continue;
        }
        // the initial melt is written on the device, ordered on the group's
        // stream behind its running steps: the scheduler does not wait
        if (elp_init_melt_device(j->lat, j->rec, j->g.L, j->spec.N, j->P, j->spec.linear ? 1 : 0, gp->s) != ELP_OK) {
            cudaFreeAsync(j->lat, gp->s);
            cudaFreeAsync(j->rec, gp->s);
            fail_job(s, j, ELP_ERR_ARG, "initial melt does not fit the box");
            continue;
        }
        for (size_t g = 0; g < s->groups.size(); g++)
            if (s->groups[g].get() == gp) j->group = (int)g;
        gp->members.push_back(j);
        gp->dirty = true;
        j->t_start = s->now();
        std::lock_guard<std::mutex> lk(s->mu);
        s->bytes_in_use += j->bytes;
        s->resident.push_back(j);
    }
    return true;
}

static bool rebuild(elp_server* s, SGroup* gp)
{
    elp_group& G = gp->G;
    // absolute steps of the members are kept in the jobs; rebuild the table
    G.jobs.clear();
    G.N.clear();
    for (size_t i = 0; i < gp->members.size(); i++) {
        SJob* j = gp->members[i];
        j->index = (int)i;
        elp_group_add(&G, j->lat, j->rec, s->d_acc, j->spec.N, j->P, j->spec.seed, j->spec.salt,
                      (uint64_t)j->done_steps, j->spec.linear ? 1 : 0);
    }
    gp->dirty = false;
    if (gp->members.empty()) return true;
    if (elp_group_commit(&G) != cudaSuccess) return false;
    if (std::get<6>(gp->key) && !G.specialised) {
        // monomer-0 moves of linear chains exist in the specialised kernels
        // only: a linear group without one refuses its jobs
        for (SJob* j : gp->members) {
            cudaFreeAsync(j->lat, gp->s);
            cudaFreeAsync(j->rec, gp->s);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->bytes_in_use -= j->bytes;
            }
            fail_job(s, j, ELP_ERR_ARG, "linear chains need a specialised kernel shape for their box");
        }
        gp->members.clear();
        G.jobs.clear();
        G.N.clear();
    }
    return true;
}

// End of a group's tick: count the steps of the jobs that ran, copy the
// state of jobs that dump or finish (on the group's stream, before its next
// tick) and hand the copies to the I/O threads, retire finished jobs.
static bool complete_tick(elp_server* s, SGroup* gp, size_t gi)
{
    const int64_t Q = s->o.quantum;
    std::vector<SJob*> done;
    for (SJob* j : gp->running) {
        j->done_steps += Q;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->moves_done += (double)Q * j->spec.N * j->P;
        }
        if (j->abort.load()) {
            // an earlier dump failed: end the job (its status is set); the
            // marker reaches the I/O threads after its queued snapshots
            Snap sn;
            sn.job = j;
            sn.step = j->done_steps;
            sn.final = true;
            sn.abort = true;
            j->pending++;
            s->io_busy++;
            {
                std::lock_guard<std::mutex> lk(s->io_mu);
                s->io_q.push_back(sn);
            }
            s->io_cv.notify_one();
            done.push_back(j);
            continue;
        }
        const bool fin = j->done_steps >= j->nsteps;
        const bool dump = j->dump_interval > 0 && j->done_steps % j->dump_interval == 0;
        if (dump || fin) {
            Snap sn;
            sn.job = j;
            sn.step = j->done_steps;
            sn.final = fin;
            const size_t S = (size_t)j->g.L * j->g.L * j->g.L;
            if (cudaMallocAsync((void**)&sn.d_lat, S * 4, gp->s) != cudaSuccess ||
                cudaMallocAsync((void**)&sn.d_rec, (size_t)j->P * ELP_REC_WORDS * 4, gp->s) != cudaSuccess ||
                cudaEventCreateWithFlags(&sn.ready, cudaEventDisableTiming) != cudaSuccess) {
                s->fatal = ELP_ERR_NOMEM;
                s->fatal_msg = "snapshot allocation failed";
                return false;
            }
            cudaMemcpyAsync(sn.d_lat, j->lat, S * 4, cudaMemcpyDeviceToDevice, gp->s);
            cudaMemcpyAsync(sn.d_rec, j->rec, (size_t)j->P * ELP_REC_WORDS * 4, cudaMemcpyDeviceToDevice, gp->s);
            cudaEventRecord(sn.ready, gp->s);
            if (dump) j->dumps++;
            j->pending++;
            s->io_busy++;
            {
                std::lock_guard<std::mutex> lk(s->io_mu);
                s->io_q.push_back(sn);
            }
            s->io_cv.notify_one();
        }
        if (fin) done.push_back(j);
    }
    for (SJob* j : done) {
        cudaFreeAsync(j->lat, gp->s);
        cudaFreeAsync(j->rec, gp->s);
        for (size_t i = 0; i < gp->members.size(); i++)
            if (gp->members[i] == j) {
                gp->members.erase(gp->members.begin() + (long)i);
                break;
            }
        gp->dirty = true;
        std::lock_guard<std::mutex> lk(s->mu);
        s->bytes_in_use -= j->bytes;
    }
    gp->running.clear();
    // a domain whose monomer-0 runs outgrew its label table stops the server
    // (the flags were copied to pinned memory behind the tick's launches)
    const uint32_t flag = s->h_err[gi];
    if (flag) {
        s->fatal = ELP_ERR_STATE;
        s->fatal_msg = "a domain held more monomer-0 runs than its label table";
        return false;
    }
    return true;
}

static void scheduler(elp_server* s)
{
    cudaSetDevice(s->o.device);
    const int64_t Q = s->o.quantum;
    for (;;) {
        if (!admit(s)) break;
        bool active = false, progressed = false;
        for (size_t gi = 0; gi < s->groups.size() && !s->fatal; gi++) {
            SGroup* gp = s->groups[gi].get();
            if (gp->busy) {
                const cudaError_t q = cudaEventQuery(gp->ev);
                if (q == cudaErrorNotReady) {
                    active = true;
                    continue;
                }
                gp->busy = false;
                progressed = true;
                if (q != cudaSuccess) {
                    s->fatal = ELP_ERR_CUDA;
                    s->fatal_msg = "tick failed";
                    break;
                }
                if (!complete_tick(s, gp, gi)) break;
            }
            if (gp->members.empty()) continue;
            if (gp->dirty && !rebuild(s, gp)) {
                s->fatal = ELP_ERR_CUDA;
                s->fatal_msg = "group rebuild failed";
                break;
            }
            if (gp->members.empty()) continue;   // its jobs were refused
            gp->running = gp->members;
            if (elp_group_run(&gp->G, Q) != cudaSuccess ||
                cudaMemcpyAsync(s->h_err + gi, s->d_err + 4 * gi, sizeof(uint32_t), cudaMemcpyDeviceToHost, gp->s) !=
                    cudaSuccess ||
                cudaEventRecord(gp->ev, gp->s) != cudaSuccess) {
                s->fatal = ELP_ERR_CUDA;
                s->fatal_msg = "launch failed";
                break;
            }
            gp->busy = true;
            active = progressed = true;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->resident.clear();
            for (auto& gp : s->groups)
                for (SJob* j : gp->members) s->resident.push_back(j);
        }
        if (s->fatal) break;
        if (!active) {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop.load() && s->queue.empty()) break;
            s->cv.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    // let the last ticks end before the jobs are failed or the groups freed
    for (auto& gp : s->groups)
        if (gp->busy) cudaEventSynchronize(gp->ev);
    if (s->fatal) {
        // the I/O threads may still hold snapshots of resident jobs: let them
        // finish (bounded) before the jobs are handed back
        for (int i = 0; i < 60000 && s->io_busy.load() > 0; i++)
            std::this_thread::sleep_for(std::chrono::milliseconds(1));
        std::lock_guard<std::mutex> lk(s->mu);
        for (SJob* j : s->resident) {
            j->status = s->fatal;
            j->error = s->fatal_msg;
            j->t_done = s->now();
            s->finished.push_back(j);
            s->completed++;
        }
        s->resident.clear();
        for (SJob* j : s->queue) {
            j->status = s->fatal;
            j->error = s->fatal_msg;
            s->finished.push_back(j);
            s->completed++;
        }
        s->queue.clear();
        s->cv_done.notify_all();
    }
}

extern "C" void elp_server_default_opts(elp_server_opts* o)
{
    memset(o, 0, sizeof(*o));
    o->device = 0;
    o->hbm_budget = 150ull << 30;
    o->quantum = 100;
    o->io_threads = 4;
    o->max_jobs = 4096;
}

extern "C" elp_status elp_server_create(const elp_server_opts* opts, elp_server** out)
{
    if (!opts || !out) return elp_fail(ELP_ERR_ARG, "null argument");
    *out = nullptr;
    if (opts->quantum < 1 || opts->io_threads < 1 || opts->max_jobs < 1)
        return elp_fail(ELP_ERR_ARG, "quantum, io_threads and max_jobs must be positive");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return elp_fail(ELP_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (opts->device < 0 || opts->device >= ndev) return elp_fail(ELP_ERR_ARG, "device %d not present", opts->device);
    ELP_CUDA_TRY(cudaSetDevice(opts->device));
    elp_server* s = new (std::nothrow) elp_server();
    if (!s) return elp_fail(ELP_ERR_NOMEM, "host allocation failed");
    s->o = *opts;
    s->t0 = std::chrono::steady_clock::now();
    if (cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, opts->device) != cudaSuccess) s->nsm = 148;
    // jobs and snapshots come and go through cudaMallocAsync: keep freed
    // blocks in this process's pool instead of unmapping them at every
    // synchronisation and mapping them again for the next job
    {
        cudaMemPool_t pool;
        uint64_t keep = UINT64_MAX;
        if (cudaDeviceGetDefaultMemPool(&pool, opts->device) == cudaSuccess)
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    uint8_t tab[4096];
    elp_build_table(tab);
    if (cudaMalloc((void**)&s->d_table, 4096) != cudaSuccess || cudaMalloc((void**)&s->d_err, 64 * 16) != cudaSuccess ||
        cudaMallocHost((void**)&s->h_err, 64 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc((void**)&s->d_acc, 8) != cudaSuccess ||
        cudaMemcpy(s->d_table, tab, 4096, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(s->d_err, 0, 64 * 16) != cudaSuccess || cudaMemset(s->d_acc, 0, 8) != cudaSuccess) {
        cudaFree(s->d_table); cudaFree(s->d_err); cudaFree(s->d_acc); cudaFreeHost(s->h_err);
        delete s;
        return elp_fail(ELP_ERR_CUDA, "server set-up failed");
    }
    memset(s->h_err, 0, 64 * sizeof(uint32_t));
    for (int i = 0; i < opts->io_threads; i++) s->io_threads.emplace_back(io_worker, s);
    s->sched = std::thread(scheduler, s);
    *out = s;
    return ELP_OK;
}

extern "C" elp_status elp_server_submit(elp_server* s, const elp_job_spec* spec, int64_t nsteps, int64_t dump_interval,
                                        const char* dump_dir, uint64_t* id)
{
    if (!s || !spec) return elp_fail(ELP_ERR_ARG, "null argument");
    if (nsteps < 1) return elp_fail(ELP_ERR_ARG, "a job needs at least one step");
    const int64_t Q = s->o.quantum;
    if (nsteps % Q) return elp_fail(ELP_ERR_ARG, "steps must be a multiple of the quantum (%lld)", (long long)Q);
    if (dump_interval < 0 || (dump_interval && dump_interval % Q))
        return elp_fail(ELP_ERR_ARG, "dump interval must be a multiple of the quantum (%lld)", (long long)Q);
    SJob* j = new (std::nothrow) SJob();
    if (!j) return elp_fail(ELP_ERR_NOMEM, "host allocation failed");
    j->spec = *spec;
    j->spec.steps_per_launch = (int32_t)Q;
    elp_status st = elp_resolve_spec(&j->spec, &j->P, &j->g);
    if (st) {
        delete j;
        return st;
    }
    j->nsteps = nsteps;
    j->dump_interval = dump_interval;
    if (dump_dir && dump_dir[0]) {
        j->dir = dump_dir;
        mkdir(dump_dir, 0755);
    }
    const size_t S = (size_t)j->g.L * j->g.L * j->g.L;
    j->bytes = 2 * (S * 4 + (size_t)j->P * ELP_REC_WORDS * 4);  // resident state + one snapshot
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop.load()) {
        delete j;
        return elp_fail(ELP_ERR_STATE, "server is shutting down");
    }
    j->id = s->next_id++;
    j->t_submit = s->now();
    s->queue.push_back(j);
    s->submitted++;
    s->cv.notify_all();
    if (id) *id = j->id;
    return ELP_OK;
}

extern "C" elp_status elp_server_poll(elp_server* s, elp_job_result* out, int32_t cap, int32_t* n)
{
    if (!s || !n || (cap > 0 && !out)) return elp_fail(ELP_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    int k = 0;
    while (k < cap && !s->finished.empty()) {
        SJob* j = s->finished.front();
        s->finished.erase(s->finished.begin());
        elp_job_result& r = out[k++];
        memset(&r, 0, sizeof(r));
        r.id = j->id;
        r.status = j->status;
        r.integrity = j->integrity;
        r.t_submit = j->t_submit;
        r.t_start = j->t_start;
        r.t_done = j->t_done;
        r.steps = (uint64_t)j->done_steps;
        r.moves = (uint64_t)j->done_steps * (uint64_t)j->spec.N * (uint64_t)j->P;
        r.dumps = j->dumps;
        r.checksum = j->checksum;
        r.L = j->g.L;
        r.N = j->spec.N;
        r.P = j->P;
        delete j;
    }
    *n = k;
    return ELP_OK;
}

extern "C" elp_status elp_server_get_stats(elp_server* s, elp_server_stats* st)
{
    if (!s || !st) return elp_fail(ELP_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->queued = s->queue.size();
    st->resident = s->resident.size();
    st->bytes_in_use = s->bytes_in_use;
    st->moves = s->moves_done;
    st->clock = s->now();
    st->fatal = s->fatal;
    return ELP_OK;
}

extern "C" elp_status elp_server_drain(elp_server* s, double timeout_s)
{
    if (!s) return elp_fail(ELP_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                  [&] { return s->completed == s->submitted || s->fatal; });
    if (s->fatal) return elp_fail(s->fatal, "server stopped: %s", s->fatal_msg.c_str());
    if (!ok) return elp_fail(ELP_ERR_BUSY, "jobs still running after %.1f s", timeout_s);
    return ELP_OK;
}

extern "C" void elp_server_destroy(elp_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (SJob* j : s->queue) delete j;
        s->queue.clear();
        s->cv.notify_all();
    }
    // finish the jobs already on the GPU, then stop
    while (true) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->resident.empty() || s->fatal) break;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(5));
    }
    if (s->sched.joinable()) s->sched.join();
    // the last snapshots: each takes a walk, a check and a file write; give
    // them a generous bound.  If the I/O threads do not finish in time they
    // are left running with the server's host state (leaked, not freed under
    // them) and only the call returns.
    bool io_done = false;
    for (int i = 0; i < 300000 && !(io_done = s->io_busy.load() == 0); i++)
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
    {
        std::lock_guard<std::mutex> lk(s->io_mu);
        s->io_stop = true;
    }
    s->io_cv.notify_all();
    if (!io_done) {
        elp_fail(ELP_ERR_BUSY, "server I/O threads still busy after 300 s; server state leaked");
        for (auto& t : s->io_threads) t.detach();
        return;
    }
    for (auto& t : s->io_threads) t.join();
    cudaSetDevice(s->o.device);
    for (auto& gp : s->groups) {
        cudaStreamSynchronize(gp->s);
        elp_group_free(&gp->G);
        cudaStreamDestroy(gp->s);
        cudaEventDestroy(gp->ev);
    }
    cudaFree(s->d_table); cudaFree(s->d_err); cudaFree(s->d_acc); cudaFreeHost(s->h_err);
    for (SJob* j : s->finished) delete j;
    delete s;
}
