/*
 * elp_ne_list NE_LIST -- lines for the reference analysis's ne_list for runs
 * of this engine in tiled geometries.
 *
 * The analysis looks a run up in scripts/ne_list.dat by the "Executable" of
 * its settings and its density, and reads the entanglement length Ne and the
 * time factor tFac from that line (analysis/mode_init.c:699-727).  Whole-box
 * runs write "Executable = efpol": their dynamics are efpol's.  Tiled runs
 * write elp_<tx>x<ty>x<tz>: their equilibrium is efpol's but their clock runs
 * slower by the factor f of elp_time_factor, so for every "efpol <density>
 * <Ne> <prefactor> <tFac> <moves>" line of NE_LIST this prints, per tile
 * shape with a measured f, "elp_<shape> <density> <Ne> <prefactor> <tFac/f>
 * 0" (the last column, the reference's informal speed in M moves/s, is not
 * read by the analysis).  f was measured at density 1.2; it is applied at
 * every density.  Append the output to the ne_list the analysis reads:
 *
 *     bin/elp_ne_list scripts/ne_list.dat >> scripts/ne_list.dat
 *
 * Exit codes: 0 ok, 192 NE_LIST cannot be read.
 */
#include <stdio.h>
#include <string.h>

#include "elp.h"

static const int kShapes[][3] = {{32, 32, 32}, {32, 32, 16}, {32, 16, 16}, {16, 16, 16}, {48, 24, 24}};

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s NE_LIST\n", argv[0]);
        return 192;
    }
    FILE* f = fopen(argv[1], "r");
    if (!f) {
        fprintf(stderr, "%s: cannot read %s\n", argv[0], argv[1]);
        return 192;
    }
    char line[1024];
    while (fgets(line, sizeof(line), f)) {
        char name[64];
        double density, ne, pre, tfac;
        if (sscanf(line, "%63s %lf %lf %lf %lf", name, &density, &ne, &pre, &tfac) != 5) continue;
        if (strcmp(name, "efpol") != 0) continue;
        for (size_t i = 0; i < sizeof(kShapes) / sizeof(kShapes[0]); i++) {
            const double tf = elp_time_factor(0, kShapes[i][0], kShapes[i][1], kShapes[i][2]);
            if (tf <= 0) continue;
            printf("elp_%dx%dx%d %.1f %.0f %.2f %.3f 0\n", kShapes[i][0], kShapes[i][1], kShapes[i][2], density, ne, pre,
                   tfac / tf);
        }
    }
    fclose(f);
    return 0;
}
