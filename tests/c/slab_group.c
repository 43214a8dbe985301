/*
 * slab_group.c -- one solve over a group of GPUs from C, the way a Fortran
 * DNS would call it: rank 0 makes the group id (the DNS would MPI_Bcast its
 * RC_SLAB_ID_BYTES bytes), every rank joins with its GPU and calls
 * rc_slab_solve with its context (p_col = number of ranks) on host arrays;
 * every rank receives the whole solution.  Here the group has one rank
 * (one GPU), so the program checks the group's path -- the library's own
 * NCCL, the field broadcast, the in-place gathers, the wall layout and the
 * host staging -- against the plain solve of the same field, bit for bit.
 *
 * usage: slab_group PARAM_H NARROWBAND_H SCRATCH_DIR   (param.h with p_col = 1)
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "radchan.h"

static int fail(const char *what, const rc_slab_comm *g) {
    char buf[512];
    if (g) rc_slab_last_error(g, buf, sizeof(buf));
    else rc_last_error(NULL, buf, sizeof(buf));
    fprintf(stderr, "slab_group: %s failed: %s\n", what, buf);
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s PARAM_H NARROWBAND_H SCRATCH_DIR\n", argv[0]);
        return 2;
    }
    rc_params p;
    if (rc_params_from_headers(argv[1], argv[2], &p)) return fail("rc_params_from_headers", NULL);
    const int nranks = 1, rank = 0;
    p.p_col = nranks;
    rc_synth_spec spec = {p.nB, p.nQ, p.nT, 300.0, 2000.0, 500.0, 10000.0, -3.0, 2.0, 1.0, 1.5, 20240601u};
    rc_table_set *ts = NULL;
    if (rc_tables_synthetic(&spec, &ts)) return fail("rc_tables_synthetic", NULL);
    if (rc_tables_write_dir(ts, argv[3])) return fail("rc_tables_write_dir", NULL);
    rc_tables_free(ts);
    ts = NULL;
    if (rc_tables_read_dir(argv[3], p.nT, p.nB, p.nQ, &ts)) return fail("rc_tables_read_dir", NULL);

    const int ni = p.imax + 2, nj = p.jmax + 2, nk = p.kmax + 2;
    const size_t nT = (size_t)ni * nj * nk;
    float *T = (float *)malloc(nT * sizeof(float));
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const double x = (i - 0.5) / p.imax;
                const double base = p.Tw[RC_WEST] + (p.Tw[RC_EAST] - p.Tw[RC_WEST]) * x;
                T[((size_t)k * nj + j) * ni + i] = (float)(base * (1.0 + 0.03 * sin(0.9 * j + 1.1 * k)));
            }

    rc_ctx *ctx = NULL;
    if (rc_create(&p, 0, &ctx)) return fail("rc_create", NULL);
    rc_tables v;
    rc_tables_view(ts, &v);
    if (rc_set_tables(ctx, &v)) return fail("rc_set_tables", NULL);

    /* the plain solve */
    const size_t nc = (size_t)p.imax * p.jmax * p.kmax, nw = (size_t)2 * p.jmax * p.kmax;
    double *q0 = (double *)calloc(nc, 8), *v0 = (double *)calloc(nc, 8);
    double *qw0 = (double *)calloc(nw, 8), *vw0 = (double *)calloc(nw, 8);
    rc_ticket t;
    if (rc_solve_async(ctx, T, 1, &t)) return fail("rc_solve_async", NULL);
    if (rc_collect(ctx, t, NULL, NULL, q0, v0, qw0, vw0)) return fail("rc_collect", NULL);

    /* the group */
    unsigned char id[RC_SLAB_ID_BYTES];
    if (rank == 0 && rc_slab_unique_id(id)) return fail("rc_slab_unique_id", NULL);
    /* (a DNS: MPI_Bcast(id, RC_SLAB_ID_BYTES, MPI_BYTE, 0, comm)) */
    rc_slab_comm *g = NULL;
    if (rc_slab_comm_create(0, nranks, rank, id, 120.0, &g)) return fail("rc_slab_comm_create", NULL);
    int kloc = 0, zstart = 0;
    if (rc_slab_range(p.kmax, nranks, rank, &kloc, &zstart)) return fail("rc_slab_range", NULL);
    double *q = (double *)calloc(nc, 8), *vv = (double *)calloc(nc, 8);
    double *qw = (double *)calloc(nw, 8), *vw = (double *)calloc(nw, 8);
    if (rc_slab_solve(g, ctx, T, q, vv, qw, vw)) return fail("rc_slab_solve", g);

    const int same = memcmp(q, q0, nc * 8) == 0 && memcmp(vv, v0, nc * 8) == 0 && memcmp(qw, qw0, nw * 8) == 0 &&
                     memcmp(vw, vw0, nw * 8) == 0;
    int nonzero = 0;
    for (size_t c = 0; c < nc && !nonzero; ++c) nonzero = q[c] != 0.0;
    printf("slab_group: %dx%dx%d, %d rank(s), slab %d planes from %d: identical %d nonzero %d\n", p.imax, p.jmax,
           p.kmax, nranks, kloc, zstart, same, nonzero);
    if (rc_slab_comm_destroy(g)) return fail("rc_slab_comm_destroy", NULL);
    rc_destroy(ctx);
    rc_tables_free(ts);
    free(T);
    free(q0);
    free(v0);
    free(qw0);
    free(vw0);
    free(q);
    free(vv);
    free(qw);
    free(vw);
    return (same && nonzero) ? 0 : 1;
}
