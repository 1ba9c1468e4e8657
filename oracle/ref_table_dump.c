/*
 * Test infrastructure (oracle): dumps the reference's own transition table.
 *
 * This driver is compiled together with the UNMODIFIED reference sources
 * cpupol/efpol_init.c, efpol_lib.c, efpol_io.c, efpol_meas.c and util/timer.c
 * (see oracle/Makefile, target `ref`).  It calls the reference's
 * SetConstants (cpupol/efpol_init.c:209) and SetTransTable
 * (cpupol/efpol_init.c:314) and writes the resulting LookupTables
 * (cpupol/efpol.h:49-55) as raw little-endian arrays:
 *   4096 x uint32 transTable, 4096 x int32 addOccup, 4096 x int32 remOccup.
 *
 * usage: ref_table_dump <model: 1=sl_equal 2=sl_double 4=sl_quad> <BL> <out>
 */
#define IS_MAIN
#include "efpol.h"

int main(int argc, char** argv){
	if(argc < 4){
		fprintf(stderr, "usage: %s model BL out\n", argv[0]);
		return 1;
	}
	int model = atoi(argv[1]);
	int bl = atoi(argv[2]);
	Constants con;
	SetConstants(&con, bl);
	SetTransTable(&con, model);
	FILE* f = fopen(argv[3], "wb");
	if(!f) return 2;
	fwrite(tab.transTable, sizeof(unsigned int), 4096, f);
	fwrite(tab.addOccup, sizeof(int), 4096, f);
	fwrite(tab.remOccup, sizeof(int), 4096, f);
	fclose(f);
	return 0;
}
