/*
 * efpol_ring / efpol_lin -- drop-in replacements of the reference's CPU
 * programs efpol_ring and efpol_lin (cpupol/efpol.c:4-114 built for rings
 * or linear chains) running the ELP sweep on the GPU.
 *
 *   efpol_ring SEED DIR DENSITY TIME INTERVAL NMONO DBLSTEP L MODEL
 *
 * Same arguments (do_run.sh:343), same output tree and file names.  NMONO
 * and L are the final ring length and box; with DBLSTEP = k the run starts
 * at NMONO / 8^k monomers in a box of L / 2^k (rounded up to a power of two,
 * efpol.c:41-58) and doubles k times (cpupol/efpol.c:84-101).  Every level
 * i writes DIR/N_<N_i>/t=<t>_dev=0.res every INTERVAL steps from t=0, a last
 * file at ceil(TIME/INTERVAL)*INTERVAL, and DIR/N_<N_i>/simulation_settings.txt
 * with the keys of cpupol/efpol_io.c:111-140.  The ring count is GetNPol of
 * the first level.  The MC steps run on the GPU; the doubling between levels
 * is elp_double_chains on the host.  Exit codes as efpol: 0 ok, 192
 * integrity failure, 193 unknown or unsupported model (sl_equal only), 212
 * melt too small to halve.  With ELP_PTL=1 in the environment the per-ring
 * time series DIR/N_<N_i>/ptl/pol=<p>_dev=0.res are written during the run
 * as well.  A whole-box level writes "Executable = efpol": its dynamics are
 * efpol's single-monomer dynamics (same move table and attempt rate).  A
 * tiled level (L > 32) writes elp_<tx>x<ty>x<tz>, its tile shape: the tile
 * walls slow its clock by elp_time_factor, and bin/elp_ne_list gives the
 * analysis the matching time factor.
 */
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "elp.h"
#include "elp_dump.h"

/* Built twice: efpol_ring, and with ELP_LINEAR_CHAINS as efpol_lin, the
 * reference's efpol built with POL_TYPE=POL_LIN (cpupol/Makefile:13-14). */
#ifdef ELP_LINEAR_CHAINS
#define PROG "efpol_lin"
#define LINEAR 1
#else
#define PROG "efpol_ring"
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

static int die(elp_status st, int code)
{
    fprintf(stderr, PROG ": %s: %s\n", elp_status_string(st), elp_last_error());
    return code;
}

int main(int argc, char** argv)
{
    unsigned seed = 37249131u;
    const char* dir = "./data/test";
    double density = 1.0;
    long tmax = 1000, interval = 100;
    int nmono = 4, dbl = 0, lstart = 16;
    const char* model = "sl_quad";
    if (argc <= 8) {
        printf("In testing mode, using defaults\n");
    } else {
        seed = (unsigned)strtoul(argv[1], 0, 10);
        dir = argv[2];
        density = atof(argv[3]);
        tmax = (long)atof(argv[4]);
        interval = (long)atof(argv[5]);
        nmono = atoi(argv[6]);
        dbl = atoi(argv[7]);
        lstart = atoi(argv[8]);
        model = argc > 9 ? argv[9] : "";
    }
    if (strcmp(model, "sl_equal") != 0) {
        if (strcmp(model, "sl_double") && strcmp(model, "sl_quad")) {
            printf("Unknown polymer model, aborting!\n");
            return 193;
        }
        fprintf(stderr, PROG ": model %s is not provided (sl_equal only)\n", model);
        return 193;
    }
    if (LINEAR && dbl != 0) {
        /* DoubleLattice doubles rings only (linear chains would keep an end marker inside the chain) */
        fprintf(stderr, PROG ": hierarchical doubling (DBLSTEP > 0) is provided for rings only\n");
        return 193;
    }
    if (dbl < 0 || dbl > 6) {
        fprintf(stderr, PROG ": DBLSTEP must be in [0, 6]\n");
        return 193;
    }
    for (int i = 0; i < dbl; i++) {
        lstart /= 2;
        nmono /= 8;
    }
    if (lstart < 2 || nmono < 2) {
        printf("Error polymer or lattice too small\n");
        return 212;
    }
    if (interval < 1 || tmax < 1) {
        fprintf(stderr, PROG ": TIME and INTERVAL must be positive\n");
        return 212;
    }
    int bl;
    for (bl = 0; bl <= 9; bl++)
        if ((1 << bl) >= lstart) break;
    const int L0 = 1 << bl;

    char sub[4096], file[4200];
    for (int i = 0, n = nmono; i <= dbl; i++, n *= 8) {
        snprintf(sub, sizeof(sub), "%s/N_%d", dir, n);
        if (mkdir_p(sub)) {
            fprintf(stderr, PROG ": cannot create %s\n", sub);
            return 192;
        }
    }
    int32_t P = 0;
    int32_t* start = NULL;
    uint8_t* bonds = NULL;
    const long ndump = (tmax - 1) / interval + 2;  /* t = 0, INTERVAL, ..., last */
    for (int lev = 0; lev <= dbl; lev++) {
        int L = L0 << lev, N = nmono;
        for (int i = 0; i < lev; i++) N *= 8;
        elp_job_spec spec;
        elp_default_spec(&spec);
        spec.L = L;
        spec.N = N;
        spec.P = P;            /* 0 on the first level: GetNPol of the density */
        spec.density = density;
        spec.seed = seed;
        spec.salt = (uint32_t)lev;
        spec.steps_per_launch = interval < 100 ? (int)interval : 100;
        spec.linear = LINEAR;
        elp_ctx* ctx = NULL;
        elp_status st = elp_create(&spec, &ctx);
        if (st) return die(st, 192);
        elp_info info;
        elp_get_info(ctx, &info);
        P = info.P;
        st = lev == 0 ? elp_init_melt(ctx) : elp_load_chains(ctx, start, bonds, 0);
        if (st) return die(st, 192);
        int32_t code = 0;
        if ((st = elp_check(ctx, &code)) || code) {
            elp_destroy(ctx);
            return 192;
        }
        snprintf(sub, sizeof(sub), "%s/N_%d", dir, N);
        elp_dumper dumper;
        if ((st = elp_dumper_open(&dumper, ctx, sub, (int32_t)ndump))) return die(st, 192);
        const double total = (double)tmax * N * P;
        double done = 0;
        for (long t = 0; t < tmax; t += interval) {
            snprintf(file, sizeof(file), "%s/t=%ld_dev=0.res", sub, t);
            if ((st = elp_dumper_write(&dumper, ctx, file))) return die(st, 192);
            double t0 = now_s();
            if ((st = elp_run(ctx, interval)) || (st = elp_sync(ctx))) return die(st, 192);
            double dt = now_s() - t0;
            done += (double)interval * N * P;
            printf("\b \b\b \b\rrun = 1/1, L=%d, [%.1lf%%] at %.2lf M/s", L, 100 * done / total,
                   1e-6 * interval * N * P / (dt > 0 ? dt : 1e-9));
            fflush(NULL);
        }
        snprintf(file, sizeof(file), "%s/t=%ld_dev=0.res", sub, ((tmax - 1) / interval + 1) * interval);
        if ((st = elp_dumper_write(&dumper, ctx, file))) return die(st, 192);
        if ((st = elp_check(ctx, &code)) || code) {
            elp_destroy(ctx);
            return 192;
        }
        if (lev < dbl) {
            /* DoubleLattice: the next level starts from the doubled final state */
            int32_t* s2 = (int32_t*)malloc((size_t)P * 3 * sizeof(int32_t));
            uint8_t* b2 = (uint8_t*)malloc((size_t)P * (size_t)N * 8);
            free(start);
            free(bonds);
            start = (int32_t*)malloc((size_t)P * 3 * sizeof(int32_t));
            bonds = (uint8_t*)malloc((size_t)P * (size_t)N);
            if (!s2 || !b2 || !start || !bonds) return die(ELP_ERR_NOMEM, 192);
            if ((st = elp_fetch_chains(ctx, start, bonds))) return die(st, 192);
            if ((st = elp_double_chains(L, N, P, start, bonds, s2, b2))) return die(st, 192);
            free(start);
            free(bonds);
            start = s2;
            bonds = b2;
        }
        /* WriteSimulationSettings, cpupol/efpol_io.c:111-140 */
        snprintf(file, sizeof(file), "%s/simulation_settings.txt", sub);
        FILE* f = fopen(file, "w");
        if (!f) {
            elp_destroy(ctx);
            return 192;
        }
        fprintf(f, "Start_seed = %u\n", seed);
        fprintf(f, "Length = %i\n", N);
        fprintf(f, LINEAR ? "Polytype = lin\n" : "Polytype = ring\n");
        fprintf(f, "Density = %lf\n", density);
        fprintf(f, "Latsize = %i\n", L);
        fprintf(f, "Start_polysize = %i\n", nmono);
        fprintf(f, "Double_step = %i\n", lev);
        fprintf(f, "Interval = %li\n", interval);
        fprintf(f, "Equilibrated = 0\n");
        fprintf(f, "Npol = %i\n", P);
        fprintf(f, "Polymodel = sl_equal\n");
        if (info.periodic)
            fprintf(f, "Executable = efpol\n");
        else
            fprintf(f, "Executable = elp_%dx%dx%d\n", info.tile[0], info.tile[1], info.tile[2]);
        fclose(f);
        if ((st = elp_dumper_close(&dumper))) return die(st, 192);
        elp_destroy(ctx);
    }
    free(start);
    free(bonds);
    printf("\nFinal sanity check succeeded\n");
    return 0;
}
