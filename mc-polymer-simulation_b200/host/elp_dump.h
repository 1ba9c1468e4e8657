/*
 * elp_dump.h -- one dump of the drop-in programs: the melt's invariants are
 * checked (elp_fetch_checked: one ring walk and one site scan, efpol's codes
 * 3/4) and the TUV file is written; when the environment sets ELP_PTL=1, the
 * same state also goes out as one more line of every ring's per-ring time
 * series (SAMPLE_DIR/ptl/pol=<p>_dev=0.res, the files the reference's
 * analysis/create_ptl.c builds afterwards from the TUV dumps).  The PTL files
 * are closed after simulation_settings.txt is written, so create_ptl finds
 * them up to date and skips its transposition pass.  A dump whose check
 * fails writes nothing and returns ELP_ERR_INTEGRITY (the programs then exit
 * 192, as efpol does when CheckIntegrity fails, cpupol/efpol.c:68-111).
 */
#ifndef ELP_DUMP_H
#define ELP_DUMP_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "elp.h"

typedef struct elp_dumper {
    elp_ptl* ptl;
    int32_t* start;
    uint8_t* bonds;
    char* text;
    size_t cap;
    elp_info info;
} elp_dumper;

static int elp_ptl_requested(void)
{
    const char* e = getenv("ELP_PTL");
    return e && e[0] == '1' && e[1] == '\0';
}

/* ntime: the number of dumps the run writes into sample_dir (0: no PTL
 * files, e.g. for a resumed run, which could not cover its earlier dumps). */
static elp_status elp_dumper_open(elp_dumper* d, elp_ctx* ctx, const char* sample_dir, int32_t ntime)
{
    memset(d, 0, sizeof(*d));
    elp_status st = elp_get_info(ctx, &d->info);
    if (st) return st;
    d->start = (int32_t*)malloc((size_t)d->info.P * 3 * sizeof(int32_t));
    d->bonds = (uint8_t*)malloc((size_t)d->info.P * (size_t)d->info.N);
    if (!d->start || !d->bonds) return ELP_ERR_NOMEM;
    if (ntime <= 0 || !elp_ptl_requested()) return ELP_OK;
    return elp_ptl_open(sample_dir, 0, d->info.P, d->info.N, ntime, 0, &d->ptl);
}

static elp_status elp_dumper_write(elp_dumper* d, elp_ctx* ctx, const char* file)
{
    const elp_info* i = &d->info;
    int32_t code = 0;
    elp_status st = elp_fetch_checked(ctx, d->start, d->bonds, &code);
    if (st) return st;
    if (code) {
        fprintf(stderr, "integrity check failed before writing %s (code %d)\n", file, code);
        return ELP_ERR_INTEGRITY;
    }
    size_t len = 0;
    if ((st = elp_format_tuv(i->L, i->N, i->P, d->start, d->bonds, NULL, 0, &len))) return st;
    if (len + 1 > d->cap) {
        free(d->text);
        d->text = (char*)malloc(len + 1);
        d->cap = d->text ? len + 1 : 0;
        if (!d->text) return ELP_ERR_NOMEM;
    }
    if ((st = elp_format_tuv(i->L, i->N, i->P, d->start, d->bonds, d->text, d->cap, &len))) return st;
    FILE* f = fopen(file, "wb");
    if (!f) return ELP_ERR_IO;
    const int ok = fwrite(d->text, 1, len, f) == len;
    if (fclose(f) || !ok) return ELP_ERR_IO;
    return d->ptl ? elp_ptl_append(d->ptl, d->start, d->bonds) : ELP_OK;
}

static elp_status elp_dumper_close(elp_dumper* d)
{
    elp_status st = d->ptl ? elp_ptl_close(d->ptl) : ELP_OK;
    free(d->start);
    free(d->bonds);
    free(d->text);
    memset(d, 0, sizeof(*d));
    return st;
}
#endif
