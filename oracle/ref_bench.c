/*
 * ref_bench.c -- TEST INFRASTRUCTURE ONLY (CPU baseline driver).
 *
 * Compiled together with the UNMODIFIED reference sources (oracle/Makefile,
 * target `ref`).  Sets up exactly what the reference's main does
 * (cpupol/efpol.c:49-68: ConfigInit, CSInit, SetTransTable, CreatePolymers)
 * and times the reference's own DoMCStep (cpupol/efpol_lib.c:122) with a
 * monotonic clock, excluding file output and the trailing sleep(1).
 *
 * usage: ref_bench L N density seed steps [tuv]
 * With a TUV file the melt is read by the reference's own ReadLatticeFile
 * (cpupol/efpol_io.c:3-47) instead of built by CreatePolymers: the timed
 * steps then start from that configuration (e.g. a relaxed melt).
 * Prints {"moves_per_s":..,"seconds":..,"moves":..,"integrity":..}.
 */
#define IS_MAIN
#include "efpol.h"
#include <time.h>

int main(int argc, char** argv)
{
    if (argc < 6) { fprintf(stderr, "usage: %s L N density seed steps [tuv]\n", argv[0]); return 1; }
    int L = atoi(argv[1]), N = atoi(argv[2]);
    cfg.density = atof(argv[3]);
    cfg.seed = (uint)strtoul(argv[4], 0, 10);
    long steps = atol(argv[5]);
    cfg.polModel = SL_EQUAL;
    cfg.interval = steps;
    cfg.dir = "/tmp";
    Seed(cfg.rngState, cfg.seed);
    int bl;
    for (bl = 0; bl <= 9; bl++) if ((1 << bl) >= L) break;
    int nPol = MAX(GetNPol(cfg.density, N, (1 << bl) * (1 << bl) * (1 << bl)), 1);
    CSInit(cs, bl, N, nPol, NULL);
    SetTransTable(&cs[0].con, cfg.polModel);
    if (argc > 6) {
        int rc = ReadLatticeFile(cs, argv[6]);
        if (rc) { fprintf(stderr, "%s: ReadLatticeFile(%s) failed (%d)\n", argv[0], argv[6], rc); return 2; }
        rc = CheckIntegrity(cs);
        if (rc) { fprintf(stderr, "%s: %s fails the integrity check (%d)\n", argv[0], argv[6], rc); return 192; }
    } else {
        CreatePolymers(&cfg, cs);
    }
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    DoMCStep(cs, steps);
    clock_gettime(CLOCK_MONOTONIC, &b);
    double sec = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
    double moves = (double)steps * N * nPol;
    int rc = CheckIntegrity(cs);
    printf("{\"moves_per_s\": %.6g, \"seconds\": %.6g, \"moves\": %.6g, \"integrity\": %d}\n", moves / sec, sec, moves, rc);
    return rc ? 192 : 0;
}
