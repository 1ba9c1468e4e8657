/*
 * gpupol3_cuda_ring -- drop-in replacement of the reference's GPU program
 * gpupol3_cuda_ring / gpupol2_cuda_ring (gpupol2/gpupol2.c:14-70).
 *
 *   gpupol3_cuda_ring NMONO TIME SEED DIR DENSITY FASTEQ INTERVAL LT LU LV [EQUIL] [DBL]
 *
 * Same arguments (do_run.sh:355), same outputs: DIR/t=0_dev=0.res on a fresh
 * start, then DIR/t=<t>_dev=0.res after every INTERVAL steps, and
 * DIR/simulation_settings.txt (gpupol2/gpupol_io.c:31-77 keys).  A directory
 * that already holds t= files is resumed from the newest one, as gpupol does
 * (gpupol2/gpupol_init.c:96-133), and TIME more steps are run; unlike gpupol
 * (which bumps the seed) the resumed run continues the same random stream,
 * so it is bit-identical to an uninterrupted run.  The box must be cubic
 * (LT = LU = LV).  The initial melt is the efpol one and the dynamics are
 * efpol's single-monomer dynamics, hence "Executable = efpol" in the
 * settings of a whole-box run (the analysis picks its time factor from that
 * name); a tiled run writes elp_<tx>x<ty>x<tz>, its tile shape, whose
 * slower clock (elp_time_factor) bin/elp_ne_list gives the analysis.  With
 * ELP_PTL=1 in the environment a fresh run also writes the per-ring time
 * series DIR/ptl/pol=<p>_dev=0.res during the run (not on resume: those files
 * would have to cover the earlier dumps too).
 */
#include <dirent.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "elp.h"
#include "elp_dump.h"

/* Built twice: gpupol3_cuda_ring, and with ELP_LINEAR_CHAINS as
 * gpupol3_cuda_lin (do_run.sh:261-262 names the program after POL_TYPE). */
#ifdef ELP_LINEAR_CHAINS
#define PROG "gpupol3_cuda_lin"
#define LINEAR 1
#else
#define PROG "gpupol3_cuda_ring"
#define LINEAR 0
#endif

static int mkdir_p(const char* path)
{
    char buf[4096];
    size_t n = strlen(path);
    if (n == 0 || n >= sizeof(buf)) return -1;
    memcpy(buf, path, n + 1);
    for (size_t i = 1; i <= n; i++) {
        if (buf[i] == '/' || buf[i] == '\0') {
            char c = buf[i];
            buf[i] = '\0';
            if (mkdir(buf, 0755) && errno != EEXIST) return -1;
            buf[i] = c;
        }
    }
    return 0;
}

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* newest "t=<t>_dev=0.res" in dir, or -1 */
static long newest_t(const char* dir)
{
    DIR* d = opendir(dir);
    if (!d) return -1;
    long best = -1;
    struct dirent* e;
    while ((e = readdir(d))) {
        long t;
        int dev;
        if (sscanf(e->d_name, "t=%ld_dev=%d.res", &t, &dev) == 2 && dev == 0 && t > best) best = t;
    }
    closedir(d);
    return best;
}

static int die(elp_status st)
{
    fprintf(stderr, PROG ": %s: %s\n", elp_status_string(st), elp_last_error());
    return 192;
}

int main(int argc, char** argv)
{
    int nmono = 2000, fasteq = 0, equil = 0, dbl = 0;
    long tmax = 50000, interval = 100;
    unsigned seed = 239864012u;
    const char* dir = ".";
    double density = 1.0;
    int lt = 32, lu = 32, lv = 32;
    if (argc > 1) nmono = atoi(argv[1]);
    if (argc > 2) tmax = (long)atof(argv[2]);
    if (argc > 3) seed = (unsigned)strtoul(argv[3], 0, 10);
    if (argc > 4) dir = argv[4];
    if (argc > 5) density = atof(argv[5]);
    if (argc > 6) fasteq = (int)atof(argv[6]);
    if (argc > 7) interval = (long)atof(argv[7]);
    if (argc > 8) lt = atoi(argv[8]);
    if (argc > 9) lu = atoi(argv[9]);
    if (argc > 10) lv = atoi(argv[10]);
    if (argc > 11) equil = atoi(argv[11]);
    if (argc > 12) dbl = atoi(argv[12]);
    if (lt != lu || lt != lv) {
        fprintf(stderr, PROG ": only cubic boxes are provided (got %dx%dx%d)\n", lt, lu, lv);
        return 192;
    }
    if (interval < 1 || tmax < 1) {
        fprintf(stderr, PROG ": TIME and INTERVAL must be positive\n");
        return 192;
    }
    if (mkdir_p(dir)) {
        fprintf(stderr, PROG ": cannot create %s\n", dir);
        return 192;
    }
    elp_job_spec spec;
    elp_default_spec(&spec);
    spec.L = lt;
    spec.N = nmono;
    spec.density = density;
    spec.seed = seed;
    spec.steps_per_launch = interval < 100 ? (int)interval : 100;
    spec.linear = LINEAR;
    elp_ctx* ctx = NULL;
    elp_status st = elp_create(&spec, &ctx);
    if (st) return die(st);
    elp_info info;
    elp_get_info(ctx, &info);
    char file[4200];
    elp_dumper dumper;
    long cur = newest_t(dir);
    if (cur >= 0) {
        printf("Starting from t=%ld\n", cur);
        if (elp_ptl_requested()) fprintf(stderr, PROG ": ELP_PTL is ignored when resuming\n");
        snprintf(file, sizeof(file), "%s/t=%ld_dev=0.res", dir, cur);
        if ((st = elp_load_tuv(ctx, file, (uint64_t)cur))) return die(st);
        if ((st = elp_dumper_open(&dumper, ctx, dir, 0))) return die(st);
        tmax += cur;
    } else {
        cur = 0;
        if ((st = elp_init_melt(ctx))) return die(st);
        if ((st = elp_dumper_open(&dumper, ctx, dir, (int32_t)(1 + (tmax + interval - 1) / interval)))) return die(st);
        snprintf(file, sizeof(file), "%s/t=0_dev=0.res", dir);
        if ((st = elp_dumper_write(&dumper, ctx, file))) return die(st);
    }
    int32_t code = 0;
    if ((st = elp_check(ctx, &code)) || code) return code ? 192 : die(st);
    const double span = (double)(tmax - cur);
    for (; cur < tmax; cur += interval) {
        double t0 = now_s();
        if ((st = elp_run(ctx, interval)) || (st = elp_sync(ctx))) return die(st);
        double dt = now_s() - t0;
        printf("\b \b\b \b\b \b\b \r[%.1lf%%] Time elapsed = %.2f s at %.2f MF/s", 100 * (1 - (tmax - cur - interval) / span),
               dt, interval * (double)lt * lu * lv / (dt > 0 ? dt : 1e-9) / 1e6);
        fflush(stdout);
        snprintf(file, sizeof(file), "%s/t=%ld_dev=0.res", dir, cur + interval);
        if ((st = elp_dumper_write(&dumper, ctx, file))) return die(st);
    }
    printf("\nSimulation complete\n");
    if ((st = elp_check(ctx, &code)) || code) return code ? 192 : die(st);
    snprintf(file, sizeof(file), "%s/simulation_settings.txt", dir);
    FILE* f = fopen(file, "w");
    if (!f) return 192;
    fprintf(f, "Start_seed = %u\n", seed);
    fprintf(f, "Length = %i\n", nmono);
    fprintf(f, LINEAR ? "Polytype = lin\n" : "Polytype = ring\n");
    fprintf(f, "Density = %lf\n", density);
    fprintf(f, "Latsize = %i\n", lt);
    fprintf(f, "Start_polysize = %i\n", nmono);
    fprintf(f, "Double_step = %i\n", dbl);
    fprintf(f, "Interval = %li\n", interval);
    fprintf(f, "Equilibrated = %i\n", equil);
    fprintf(f, "Npol = %i\n", info.P);
    fprintf(f, "Polymodel = sl_equal\n");
    if (info.periodic)
        fprintf(f, "Executable = efpol\n");
    else
        fprintf(f, "Executable = elp_%dx%dx%d\n", info.tile[0], info.tile[1], info.tile[2]);
    fprintf(f, "Fast_equilibration = %i\n", fasteq ? 1 : 0);
    fprintf(f, "FEQ_timestep = %i\n", fasteq);
    fprintf(f, "Release = elp-b200\n");
    fclose(f);
    if ((st = elp_dumper_close(&dumper))) return die(st);
    elp_destroy(ctx);
    return 0;
}
