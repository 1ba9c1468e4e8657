/*
 * tuv2pov -- drop-in replacement of the reference's analysis/tuv2pov.c:
 *
 *   tuv2pov TUV_FILE POV_FILE [POL_ID]
 *
 * writes the chains of TUV_FILE (all of them, or chain POL_ID) as a POV-Ray
 * scene (elp_tuv_to_pov); scripts/pov3d.sh renders it with an external
 * POV-Ray.  Exit codes: 0 ok, 192 missing arguments or unreadable file (as
 * the reference), 193 POL_ID out of range.
 */
#include <stdio.h>
#include <stdlib.h>

#include "elp.h"

int main(int argc, char** argv)
{
    if (argc < 3) {
        printf("Bad number of arguments\n");
        return 192;
    }
    const int pol = argc >= 4 ? atoi(argv[3]) : -1;
    elp_status st = elp_tuv_to_pov(argv[1], argv[2], pol);
    if (st) {
        fprintf(stderr, "tuv2pov: %s: %s\n", elp_status_string(st), elp_last_error());
        return st == ELP_ERR_ARG ? 193 : 192;
    }
    return 0;
}
