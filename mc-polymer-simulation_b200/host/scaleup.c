/*
 * scaleup -- drop-in replacement of the reference's analysis/scaleup.c, the
 * doubling step do_run.sh runs between GPU levels (do_run.sh:290-330):
 *
 *   scaleup SRC_FILE DST_FILE
 *
 * writes SRC_FILE's melt in a box of twice the edge with rings eight times
 * as long (elp_scaleup_tuv), byte for byte the reference's output.  Exit
 * codes: 0 ok, 192 missing arguments or a file that cannot be read or written.
 */
#include <stdio.h>

#include "elp.h"

int main(int argc, char** argv)
{
    if (argc < 3) {
        printf("Not enough arguments\n");
        return 192;
    }
    elp_status st = elp_scaleup_tuv(argv[1], argv[2]);
    if (st) {
        fprintf(stderr, "scaleup: %s: %s\n", elp_status_string(st), elp_last_error());
        return 192;
    }
    return 0;
}
