/*
 * denise_b200 - command-line front end of the B200 P-SV path.
 *
 *     denise_b200 <parameter file .inp> [device]
 *
 * Runs the forward modelling (MODE 0) of a DENISE parameter file as the
 * reference's `denise <file.inp>` does (src/denise.c: read_par, then FD_PSV),
 * and writes the same SU seismogram files.  Exit status 0 on success, 1 with
 * the library's message on stderr otherwise (the reference's err()).
 */
#include <stdio.h>
#include <stdlib.h>

#include "denise_b200_io.h"

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s <parameter file .inp> [device]\n", argv[0]);
        return 2;
    }
    const int device = argc > 2 ? atoi(argv[2]) : 0;
    dn_inp in;
    int st = dn_inp_read(argv[1], &in);
    if (st == DN_OK && in.mode != 0) {
        fprintf(stderr, "denise_b200: MODE=%d: this command runs forward modelling (MODE=0); "
                        "FWI (MODE=1) runs as: python -m denise_b200 <par.inp> <workflow.inp>\n", in.mode);
        return 1;
    }
    if (st == DN_OK) st = dn_forward_inp(argv[1], device);
    if (st != DN_OK) {
        fprintf(stderr, "denise_b200: error %d: %s\n", st, dn_last_error());
        return 1;
    }
    return 0;
}
