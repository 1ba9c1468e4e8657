/*
 * tuv2xyz -- drop-in replacement of the reference's analysis/tuv2xyz.c:
 *
 *   tuv2xyz TUV_FILE XYZ_FILE POL_ID
 *
 * writes ring POL_ID of TUV_FILE as one "x y z" line per monomer
 * (elp_tuv_to_xyz).  Exit codes as the reference: 0 ok, 192 missing
 * arguments or unreadable file, 193 POL_ID out of range.
 */
#include <stdio.h>
#include <stdlib.h>

#include "elp.h"

int main(int argc, char** argv)
{
    if (argc < 4) {
        printf("Need two arguments!\n");
        return 192;
    }
    elp_status st = elp_tuv_to_xyz(argv[1], atoi(argv[3]), argv[2]);
    if (st) {
        fprintf(stderr, "tuv2xyz: %s: %s\n", elp_status_string(st), elp_last_error());
        return st == ELP_ERR_ARG ? 193 : 192;
    }
    return 0;
}
