/* yo_cli.c -- run the oracle end to end on a yspec parameter file and write
 * the per-receiver files as the reference does.  TEST INFRASTRUCTURE ONLY. */
#include "yo.h"
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv)
{
    if (argc < 2) { fprintf(stderr, "usage: yo_cli input.in [nthreads]\n"); return 2; }
    int nth = argc > 2 ? atoi(argv[2]) : 0;
    yo_params p;
    if (yo_read_params(argv[1], &p)) { fprintf(stderr, "can't read parameter file\n"); return 1; }
    double *out = NULL;
    int nout = 0, nr = 0;
    int rc = yo_run(argv[1], &out, &nout, &nr, nth);
    if (rc) { fprintf(stderr, "oracle stop code %d\n", rc); return rc; }
    rc = yo_write_traces(p.pref_out, out, nout, nr);
    free(out);
    yo_free_params(&p);
    return rc;
}
