/*
 * efpol_port_main.c -- TEST INFRASTRUCTURE ONLY.
 * Times the efpol restatement: `efpol_port L N density seed steps`.
 * Prints one JSON line {"moves_per_s":..,"seconds":..,"moves":..}.
 * Used by bench.py as the CPU baseline when the reference build is absent.
 */
#include "oracle.h"
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

int main(int argc, char** argv)
{
    if (argc < 6) { fprintf(stderr, "usage: %s L N density seed steps\n", argv[0]); return 1; }
    int L = atoi(argv[1]), N = atoi(argv[2]);
    double rho = atof(argv[3]);
    uint32_t seed = (uint32_t)strtoul(argv[4], 0, 10);
    long steps = atol(argv[5]);
    int P = orc_get_npol(rho, N, (long)L * L * L);
    if (P < 1) P = 1;
    orc_efpol* s = orc_efpol_new(L, N, P, ORC_POL_RING, ORC_SL_EQUAL, seed);
    orc_efpol_create(s);
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    orc_efpol_mcstep(s, steps);
    clock_gettime(CLOCK_MONOTONIC, &b);
    double sec = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
    double moves = (double)steps * N * P;
    int rc = orc_efpol_check(s);
    printf("{\"moves_per_s\": %.6g, \"seconds\": %.6g, \"moves\": %.6g, \"integrity\": %d}\n", moves / sec, sec, moves, rc);
    orc_efpol_free(s);
    return rc ? 192 : 0;
}
