/*
 * elp.h -- C ABI of the B200 Elastic Lattice Polymer (ELP) sweep engine.
 *
 * Plain C types only: a caller binds this from C (the drop-in front-ends),
 * ctypes, cgo or JNI without any C++ or torch types.
 *
 * Mapping onto the reference:
 *   elp_create + elp_init_melt   <- SimPropDefaultInit/LoadPolymers/GPULibInit/
 *                                   GPULibLoadBuffers (gpupol2/gpupol_cuda.h:6-7,
 *                                   gpupol2/gpupol_init.c:83-152) and efpol's
 *                                   CSInit/SetTransTable/CreatePolymers
 *                                   (cpupol/efpol.c:60-66, cpupol/efpol_init.c:239-424)
 *   elp_run                      <- GPULibRun(nTime) (gpupol2/gpupol_cuda.h:9) and
 *                                   DoMCStep(nTime) (cpupol/efpol_lib.c:122)
 *   elp_fetch_chains             <- GPULatticeToCPU (gpupol2/gpupol_cuda.h:11)
 *   elp_write_tuv / elp_load_tuv <- WriteLatticeFile / ReadLatticeFile
 *                                   (cpupol/efpol_io.c:3-77, gpupol2/gpupol_io.c:105-203)
 *   elp_check                    <- CheckIntegrity (cpupol/efpol_io.c:158-211)
 *   elp_destroy                  <- GPULibRelease (gpupol2/gpupol_cuda.h:8)
 *
 * Errors: every call returns an elp_status; nothing calls exit() or aborts.
 * elp_last_error() gives a message for the calling thread's last failure.
 * Threading: one host thread per context at a time.
 */
#ifndef ELP_H
#define ELP_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t elp_status;
#define ELP_OK 0
#define ELP_ERR_ARG 1         /* invalid argument or geometry */
#define ELP_ERR_CUDA 2        /* CUDA error or no CUDA device */
#define ELP_ERR_NOMEM 3       /* device or host allocation failed */
#define ELP_ERR_IO 4          /* file could not be opened / written */
#define ELP_ERR_FORMAT 5      /* TUV text malformed or does not match the job */
#define ELP_ERR_INTEGRITY 6   /* configuration violates an ELP invariant */
#define ELP_ERR_STATE 7       /* call not valid in the context's state */
#define ELP_ERR_BUSY 8        /* server/queue full or admission refused */

typedef struct elp_ctx elp_ctx;

typedef struct elp_job_spec {
    int32_t L;                /* cubic box edge (sites) */
    int32_t N;                /* monomers per ring, 3 .. 65536 (linear chains: .. 65535) */
    int32_t P;                /* rings; <= 0: round(density * L^3 / N) as GetNPol */
    double density;           /* monomers per site, used when P <= 0 */
    uint32_t seed;            /* Philox key word 0 */
    uint32_t salt;            /* Philox key word 1 (independent streams) */
    int32_t periodic;         /* -1 auto, 0 tiled domains, 1 whole box on chip */
    int32_t tile[3];          /* tiled domain edges, 0 = auto */
    int32_t ncol;             /* colour modulus, 0 = auto */
    int32_t device;           /* CUDA device ordinal */
    int32_t steps_per_launch; /* steps per kernel launch (>=1); tiled domains: a cooperative launch with a
                                 grid barrier between steps.  Any value gives the same bits. */
    int32_t kernel;           /* 0 auto (specialised when the shape has one), 1 generic */
    int32_t linear;           /* 0 ring polymers (efpol_ring), 1 linear chains (efpol_lin): the last
                               * bond of every chain is the end marker 0xf ('f' in TUV files).
                               * Linear chains need a shape with a specialised kernel. */
} elp_job_spec;

typedef struct elp_info {
    int32_t L, N, P;
    int32_t periodic, tile[3], ncol;
    int32_t domains;          /* CTAs per step */
    int32_t threads;          /* threads per CTA */
    int32_t specialised;      /* 1: a shape-specialised kernel runs this melt, 0: generic kernel */
    uint64_t smem_bytes;      /* dynamic shared memory per CTA */
    uint64_t step;            /* absolute steps done */
    uint64_t device_bytes;    /* device memory held by the context */
    int32_t linear;           /* 1: linear chains */
    uint64_t kernels;         /* kernels launched for the sweep so far (a CUDA-graph replay counts its
                                 kernels: its sweep launches and the step-counter update) */
} elp_info;

/* Fill a spec with defaults: density 1.2, auto geometry, device 0. */
void elp_default_spec(elp_job_spec* spec);

/* Create a context: validates the geometry, allocates device state, uploads
 * the transition table.  The lattice starts empty (use elp_init_melt or a
 * load call). */
elp_status elp_create(const elp_job_spec* spec, elp_ctx** out);

/* Reference initial melt (CreatePolymers): step counter reset to 0. */
elp_status elp_init_melt(elp_ctx* ctx);

/* Load rings from chain form: start[3*P] = (t,u,v) of monomer 0 in [0,L),
 * bonds[P*N] = 4-bit bond codes (TUV order).  `step` sets the absolute step
 * counter, so a run resumed from a dump continues the same random stream.
 * Only the chains are copied to the device, where the site words are built.
 * Invalid chains return ELP_ERR_INTEGRITY and leave the context with no
 * configuration loaded. */
elp_status elp_load_chains(elp_ctx* ctx, const int32_t* start, const uint8_t* bonds, uint64_t step);

/* Load a TUV file (LT/LU/LV/np/maxPolLength header, len= blocks). */
elp_status elp_load_tuv(elp_ctx* ctx, const char* path, uint64_t step);

/* Run n time steps (1 step = N*P attempted monomer moves).  Asynchronous:
 * stream-ordered on the context's stream; returns after enqueueing. */
elp_status elp_run(elp_ctx* ctx, int64_t nsteps);

/* Same as elp_run, timed with CUDA events recorded on the context's stream
 * around the launches; blocks and returns the elapsed milliseconds.  Work
 * the caller queued on the stream before (elp_stream) runs ahead of the
 * first event and is not timed. */
elp_status elp_run_timed(elp_ctx* ctx, int64_t nsteps, float* ms);

/* The context's cudaStream_t, for ordering the caller's own device work
 * (copies, cache flushes) with the context's launches.  The context owns it. */
void* elp_stream(elp_ctx* ctx);

elp_status elp_sync(elp_ctx* ctx);

/* Rebuild the rings on the device and copy them to host buffers
 * start[3*P] (int32) and bonds[P*N] (uint8).  Blocking.  The rings are
 * rebuilt by list ranking over all runs at once (boxes up to L = 512; a
 * walk along each ring above).  Returns ELP_ERR_STATE if an earlier launch
 * reported an error (as elp_sync), else ELP_ERR_INTEGRITY if a chain is
 * broken (a bond that is no lattice bond, a run leading to an empty site or
 * into another chain, a wrong monomer count); on either error the buffers'
 * contents are unspecified.  With pinned buffers the copies run
 * asynchronously behind the kernels, themselves queued behind the steps.
 * Replaces GPULatticeToCPU + the host's ring rebuild
 * (gpupol2/gpupol_cuda.cu:60, gpupol2/oclpol.c:183-376). */
elp_status elp_fetch_chains(elp_ctx* ctx, int32_t* start, uint8_t* bonds);

/* elp_fetch_chains and elp_check in one pass over the melt (one ring walk,
 * one site scan): the rings go to start[3*P] / bonds[P*N] and the integrity
 * code (0 ok, 3, 4: efpol's codes, cpupol/efpol_io.c:158-211) to *code.
 * With a non-zero code the buffers are unspecified.  The drop-in programs
 * check every dump this way (the reference checks only before and after the
 * run, cpupol/efpol.c:68,111).  Blocking. */
elp_status elp_fetch_checked(elp_ctx* ctx, int32_t* start, uint8_t* bonds, int32_t* code);

/* Write the current state as a TUV file, byte-compatible with the
 * reference's WriteLatticeFile.  Blocking. */
elp_status elp_write_tuv(elp_ctx* ctx, const char* path);

/* Integrity check on the device.  *code: 0 ok, 3 two rings share a site,
 * 4 invalid bond, broken ring, bad count or bookkeeping (efpol's codes). */
elp_status elp_check(elp_ctx* ctx, int32_t* code);

elp_status elp_get_info(const elp_ctx* ctx, elp_info* info);

/* Time factor of a domain geometry against the reference efpol's clock.
 * Tile walls reject the moves that would cross them, as gpupol's block walls
 * do (gpupol2/ringpol3.cu:58-76).  The walls move every step, so the
 * equilibrium is efpol's, but the clock runs slower: after t steps a tiled
 * melt has moved as far as efpol after f*t steps (centre-of-mass MSD).
 * f = 1 for a whole-box melt (periodic = 1); for the tile shapes the engine
 * picks, f is the value measured against reference efpol ensembles (rings of
 * N = 100 at L = 64, density 1.2, steps 15000-50000); 0 for a shape not
 * measured.  The reference records its own engines' clocks the same way, as
 * the time factor of their Executable in scripts/ne_list.dat
 * (analysis/mode_init.c:699-727): the drop-in programs name a tiled run's
 * Executable after its tile shape (elp_<tx>x<ty>x<tz>), and bin/elp_ne_list
 * prints the matching ne_list lines (efpol's Ne, its time factor / f). */
double elp_time_factor(int32_t periodic, int32_t tx, int32_t ty, int32_t tz);

/* Integrity check that allocates nothing.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc -- an application that has given
 * the whole device memory to its own pool, a process under a device-memory
 * quota, a latency-critical loop that cannot take an allocation's implicit
 * device synchronisation.  It runs the checks of elp_check on a melt the
 * caller holds on the device (d_words[L^3] site words, d_records[4*P], the
 * layout of elp_get_state) and returns the same code in *code.  Ring melts
 * only: the walk follows rings, so a melt of linear chains gets code 4 (a
 * false failure); check linear melts with elp_check.  Its scratch memory is
 * a static device array of ELP_NOALLOC_MAX_SITES visit counters and
 * ELP_NOALLOC_MAX_RINGS ring statuses (about 1.5 MB, held by every GPU that
 * loads the library until the process exits); larger melts are rejected with
 * ELP_ERR_ARG.  The first call on a device looks up the array's device
 * address once and keeps it for the life of the process; make that first
 * call before any stream capture.  A process that resets the device
 * (cudaDeviceReset) must not call this entry point again, since the module
 * may then sit at another address.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  `stream` is
 * a cudaStream_t (NULL: the default stream); the call blocks until the
 * result is on the host. */
#define ELP_NOALLOC_MAX_SITES 262144u   /* L <= 64 */
#define ELP_NOALLOC_MAX_RINGS 131072u
elp_status elp_check_noalloc(const uint32_t* d_words, const uint32_t* d_records, int32_t L, int32_t N, int32_t P,
                             void* stream, int32_t* code);

/* In-situ observables of the current state, computed on the device from the
 * site words (no ring transfer).  Per ring, positions unwrapped along the
 * ring from monomer 0's site as LoadPTL (analysis/mode_io.c:509-606) builds
 * them from a TUV line:
 *   cms_tuv[3*P]  mean (t, u, v) of the ring's monomers (ComputeTUVCMS-style
 *                 lattice units; x = t+u-v, y = t-u, z = v, lengths / sqrt(2))
 *   rg2[P]        radius of gyration squared in xyz / sqrt(2) units
 *                 (ComputeGyration, analysis/mode_compute.c:191-203)
 *   sl[P]         stored-length fraction: zero bonds / N (ComputeSL, :145-153)
 *   run_hist[nbins] over the whole melt: bin k counts occupied sites holding
 *                 k+1 monomers, the last bin those holding nbins or more
 *                 (1 <= nbins <= ELP_OBS_MAX_BINS).
 * Any output may be NULL.  Blocking.  The reference computes these offline
 * from PTL files; there is no in-situ counterpart. */
#define ELP_OBS_MAX_BINS 64
elp_status elp_observe(elp_ctx* ctx, double* cms_tuv, double* rg2, double* sl, uint64_t* run_hist, int32_t nbins);

/* Raw state: words[L^3] site words, records[4*P]. Blocking. */
elp_status elp_get_state(elp_ctx* ctx, uint32_t* words, uint32_t* records);
elp_status elp_set_state(elp_ctx* ctx, const uint32_t* words, const uint32_t* records, uint64_t step);

/* Moves accepted since creation (counted on the device).  Returns
 * ELP_ERR_STATE, with the count as it stands, if an earlier launch reported
 * an error (its steps are incomplete), as elp_sync does. */
elp_status elp_accepted(elp_ctx* ctx, uint64_t* accepted);

/* Bound of the grid-barrier waits inside tiled launches of several steps.
 * No counterpart in the reference, whose launches take one step each
 * (gpupol2/gpupol_cuda.cu:129-146).  Between two steps the CTAs of a launch
 * meet at a grid barrier; a wait gives up after `polls` polls (0: the
 * default, about a second), the launch stops there and reports
 * ELP_ERR_STATE at the next synchronising call.  The context stays usable:
 * loading a configuration (elp_init_melt, a load call, elp_set_state) clears
 * the report.  hold_block >= 0 is a test hook: that CTA of each later launch
 * never arrives at the first barrier, so every wait there runs out of polls
 * -- the failure path is tested without faulting or hanging the GPU.  -1
 * lets every CTA arrive. */
elp_status elp_debug_waits(elp_ctx* ctx, uint32_t polls, int32_t hold_block);

void elp_destroy(elp_ctx* ctx);

/* The 4096-entry transition table (dst1 | dst2<<4 per option), identical to
 * the reference's transTable & 0xff for sl_equal (cpupol/efpol_init.c:314). */
elp_status elp_transition_table(uint8_t out[4096]);

/* Format chains as TUV text.  *len receives the length (excluding NUL);
 * with buf == NULL only the length is computed. */
elp_status elp_format_tuv(int32_t L, int32_t N, int32_t P, const int32_t* start, const uint8_t* bonds,
                          char* buf, size_t cap, size_t* len);

/* Hierarchical doubling of a ring melt (efpol's DoubleLattice,
 * cpupol/efpol_init.c:114-207): box 2L, rings of 8N, same P.  start_out[3*P]
 * and bonds_out[P*8*N] receive the doubled rings.  Host only.  ELP_ERR_STATE
 * if a two-site ring finds no free sites for its rebuilt form. */
elp_status elp_double_chains(int32_t L, int32_t N, int32_t P, const int32_t* start, const uint8_t* bonds,
                             int32_t* start_out, uint8_t* bonds_out);

/* Upscaling of a ring melt's TUV file for the reference's GPU doubling runs
 * (analysis/scaleup.c, called by do_run.sh): box 2L, rings 8x longer, each
 * occupied site replaced by a seven-bond path through a 2x2x2 cube, with
 * the reference's fixed random stream, so the output file is the
 * reference's byte for byte.  Host only. */
elp_status elp_scaleup_tuv(const char* in_path, const char* out_path);

/* Ring pol_id of a TUV file as xyz text, one "x y z" line per monomer
 * walked from the origin (analysis/tuv2xyz.c).  Host only.  ELP_ERR_ARG if
 * pol_id is out of range. */
elp_status elp_tuv_to_xyz(const char* in_path, int32_t pol_id, const char* out_path);

/* The chains of a TUV file as a POV-Ray scene (analysis/tuv2pov.c): camera
 * and area light placed as the reference places them, a cylinder per link
 * and a sphere per site, coloured by chain (pol_id < 0: all chains) or along
 * the one chain pol_id.  The scene text is the reference's byte for byte.
 * Host only; ELP_ERR_ARG if pol_id >= np. */
elp_status elp_tuv_to_pov(const char* in_path, const char* out_path, int32_t pol_id);

/* ---- PTL writer --------------------------------------------------------------
 * Per-ring time series written while a run dumps: sample_dir/ptl/pol=<p>_dev=<dev>.res,
 * the files the reference's create_ptl makes afterwards from the run's TUV
 * dumps (analysis/create_ptl.c:46-115): "polId= p", "nTime= ntime", "len= N",
 * then one "t u v <bond hex string>" line per dump.  Host only: needs no
 * device.  Lines are buffered (buffer_bytes, 0 = 256 MiB) and appended to the
 * files when the buffer fills and at close. */
typedef struct elp_ptl elp_ptl;
elp_status elp_ptl_open(const char* sample_dir, int32_t dev, int32_t P, int32_t N, int32_t ntime,
                        size_t buffer_bytes, elp_ptl** out);
/* One dump: start[3*P] (t,u,v of monomer 0), bonds[P*N]; ELP_ERR_STATE after ntime dumps. */
elp_status elp_ptl_append(elp_ptl* w, const int32_t* start, const uint8_t* bonds);
/* Flush and free; ELP_ERR_STATE if the number of dumps differs from ntime. */
elp_status elp_ptl_close(elp_ptl* w);

const char* elp_status_string(elp_status s);
const char* elp_last_error(void);

/* ---- batched engine --------------------------------------------------------
 * Many independent melts (replicas, seeds, parameter sweeps) of uneven box
 * size and ring length advanced together on one GPU.  All lattices live in
 * one packed arena; melts with the same domain geometry share one kernel
 * launch and a stream, and groups of different shapes run concurrently.
 * Melts run `steps_per_launch` steps per launch: whole-box melts (L <= 32)
 * on chip, tiled melts as one cooperative launch whose CTAs meet at a grid
 * barrier between steps (in a batch of more than one group, tiled groups take
 * one step per launch, so that groups keep overlapping); tiled launches are
 * replayed from a CUDA graph.  A melt gives the same bits in a batch as alone
 * with the same spec, whatever its steps per launch.
 * The reference has no batched engine; its nearest form is one independent
 * replica per GPU (gpupol2/gpupol_init.c:8-33, gpupol2/gpupol_cuda.cu:129-146). */
typedef struct elp_batch elp_batch;

elp_status elp_batch_create(const elp_job_spec* specs, int32_t njobs, int32_t device, elp_batch** out);
int32_t elp_batch_size(const elp_batch* b);
/* Reference initial melt for every member (step 0). */
elp_status elp_batch_init_melts(elp_batch* b);
elp_status elp_batch_load_chains(elp_batch* b, int32_t job, const int32_t* start, const uint8_t* bonds,
                                 uint64_t step);
/* Advance every member by nsteps (asynchronous). */
elp_status elp_batch_run(elp_batch* b, int64_t nsteps);
/* Same, timed with CUDA events across all group streams; blocks. */
elp_status elp_batch_run_timed(elp_batch* b, int64_t nsteps, float* ms);
elp_status elp_batch_sync(elp_batch* b);
/* elp_observe for member j. */
elp_status elp_batch_observe(elp_batch* b, int32_t j, double* cms_tuv, double* rg2, double* sl, uint64_t* run_hist,
                             int32_t nbins);
elp_status elp_batch_fetch_chains(elp_batch* b, int32_t job, int32_t* start, uint8_t* bonds);
elp_status elp_batch_get_state(elp_batch* b, int32_t job, uint32_t* words, uint32_t* records);
elp_status elp_batch_check(elp_batch* b, int32_t job, int32_t* code);
elp_status elp_batch_accepted(elp_batch* b, int32_t job, uint64_t* accepted);
elp_status elp_batch_job_info(const elp_batch* b, int32_t job, elp_info* info);
void elp_batch_destroy(elp_batch* b);

/* Autotuner: times the candidate domain geometries of `in` -- the whole box
 * on chip and every tile shape that divides the box, each with 1, 10 or 100
 * steps per launch -- on `copies` copies of its initial melt run as one batch
 * for `steps` steps, and returns the fastest as an explicit spec (periodic,
 * tile, ncol, steps_per_launch filled in).  "Fastest" is the time per
 * efpol-equivalent step: the time per step divided by the geometry's clock
 * factor (elp_time_factor; 1 for the wall-free whole box), so tile walls
 * cost what they slow the melt; shapes without a measured factor are not
 * candidates.  The tile shape is part of a
 * trajectory's definition: record the returned spec and reuse it; runs of the
 * same spec give the same bits, alone or batched. */
elp_status elp_autotune(const elp_job_spec* in, int32_t copies, int32_t steps, elp_job_spec* out,
                        float* ms_per_step);

/* ---- serving loop ------------------------------------------------------------
 * Continuous batching of melt jobs on one GPU.  A scheduler thread runs ticks
 * of `quantum` steps; between ticks it admits queued jobs whose device memory
 * fits `hbm_budget`, so jobs that arrive while others run join the mix as
 * memory frees up.  Lattices stay resident between dumps; a dump is copied on
 * the device at the end of a tick and rebuilt + copied to pinned host memory
 * on a side stream while the next tick computes; host threads write the TUV
 * files `dump_dir/t=<step>_dev=0.res` (no files when dump_dir is NULL or "").
 * A job's result depends only on its spec: alone or in any mix it gives the
 * same bits (reported as a checksum of its final rings).  The reference has
 * no serving mode (one job per process, gpupol2/gpupol2.c:14-70). */
typedef struct elp_server elp_server;

typedef struct elp_server_opts {
    int32_t device;
    uint64_t hbm_budget;      /* device bytes jobs may hold (state + one snapshot each) */
    int32_t quantum;          /* steps per tick; job lengths and dump intervals are multiples */
    int32_t io_threads;       /* host threads formatting and writing TUV files */
    int32_t max_jobs;         /* resident job limit */
} elp_server_opts;

typedef struct elp_job_result {
    uint64_t id;
    int32_t status;           /* ELP_OK or the error that ended the job */
    int32_t integrity;        /* CheckIntegrity code of the final state (0 ok) */
    double t_submit, t_start, t_done;   /* seconds on the server clock */
    uint64_t steps, moves;
    uint32_t dumps;
    uint64_t checksum;        /* FNV-1a of the final start[3P] and bonds[P*N] */
    int32_t L, N, P;
} elp_job_result;

typedef struct elp_server_stats {
    uint64_t submitted, completed, queued, resident, bytes_in_use;
    double moves;             /* attempted monomer moves done so far */
    double clock;             /* server clock (s) */
    int32_t fatal;            /* non-zero: the scheduler stopped on this error */
} elp_server_stats;

void elp_server_default_opts(elp_server_opts* o);
elp_status elp_server_create(const elp_server_opts* opts, elp_server** out);
/* Queue a job: initial melt of `spec`, `nsteps` steps, a TUV dump every
 * `dump_interval` steps (0: none) and at the end.  Thread-safe.  Ring and
 * linear-chain jobs run in separate groups; a linear-chain job whose box has
 * no specialised kernel shape finishes with status ELP_ERR_ARG. */
elp_status elp_server_submit(elp_server* s, const elp_job_spec* spec, int64_t nsteps, int64_t dump_interval,
                             const char* dump_dir, uint64_t* id);
/* Move up to `cap` finished jobs' results to `out`; *n receives the count. */
elp_status elp_server_poll(elp_server* s, elp_job_result* out, int32_t cap, int32_t* n);
elp_status elp_server_get_stats(elp_server* s, elp_server_stats* st);
/* Wait until every submitted job has finished (or `timeout_s` passes). */
elp_status elp_server_drain(elp_server* s, double timeout_s);
/* Drop queued jobs, finish the ones on the GPU, stop. */
void elp_server_destroy(elp_server* s);

#ifdef __cplusplus
}
#endif
#endif
