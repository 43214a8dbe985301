/*
 * legacy_abi.c -- a compiled (C99) caller of the library, the way the
 * channel DNS calls the reference: by reference, with the trailing-underscore
 * symbols mc_gpu_ / get_results_ (src/montecarlo/mc_gpu_noint.cu:660, :876),
 * the solver configured from the reference's own param.h / NarrowBand.h and
 * the table files in ./properties-style directories.
 *
 * usage: legacy_abi PARAM_H NARROWBAND_H SCRATCH_DIR
 *
 * 1. builds the seeded synthetic tables and writes them in the reference's
 *    file formats into SCRATCH_DIR;
 * 2. points RADCHAN_PARAM_H / RADCHAN_NARROWBAND_H / RADCHAN_PROPERTIES at
 *    them and calls mc_gpu_ then get_results_ on a channel temperature field;
 * 3. solves the same field through the explicit context API (headers, table
 *    files, rc_solve_async, rc_collect);
 * 4. exits 0 when both results are identical, finite and not all zero.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "radchan.h"

static int fail(const char *what) {
    char buf[512];
    rc_last_error(NULL, buf, sizeof(buf));
    fprintf(stderr, "legacy_abi: %s failed: %s\n", what, buf);
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s PARAM_H NARROWBAND_H SCRATCH_DIR\n", argv[0]);
        return 2;
    }
    rc_params p;
    if (rc_params_from_headers(argv[1], argv[2], &p)) return fail("rc_params_from_headers");

    /* tables in the reference's file formats */
    rc_synth_spec spec = {p.nB, p.nQ, p.nT, 300.0, 2000.0, 500.0, 10000.0, -3.0, 2.0, 1.0, 1.5, 20240601u};
    rc_table_set *ts = NULL;
    if (rc_tables_synthetic(&spec, &ts)) return fail("rc_tables_synthetic");
    if (rc_tables_write_dir(ts, argv[3])) return fail("rc_tables_write_dir");
    rc_tables_free(ts);

    /* T(0:imax+1, 0:jmax+1, 0:kmax+1), i fastest: wall-to-wall profile with
     * a small perturbation; x ghosts hold 2 Tw - T1 so the face average is Tw */
    const int ni = p.imax + 2, nj = p.jmax + 2, nk = p.kmax + 2;
    const size_t nf = (size_t)ni * nj * nk;
    float *T = (float *)malloc(nf * sizeof(float));
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const double x = (i - 0.5) / p.imax;
                const double base = p.Tw[RC_WEST] + (p.Tw[RC_EAST] - p.Tw[RC_WEST]) * x;
                T[((size_t)k * nj + j) * ni + i] = (float)(base * (1.0 + 0.03 * sin(0.7 * j + 1.3 * k)));
            }
    for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j) {
            float *row = T + ((size_t)k * nj + j) * ni;
            row[0] = 2.0f * p.Tw[RC_WEST] - row[1];
            row[ni - 1] = 2.0f * p.Tw[RC_EAST] - row[ni - 2];
        }

    /* the DNS's calls: configured from the environment on the first call */
    setenv("RADCHAN_PARAM_H", argv[1], 1);
    setenv("RADCHAN_NARROWBAND_H", argv[2], 1);
    setenv("RADCHAN_PROPERTIES", argv[3], 1);
    const int kloc = p.kmax / p.p_col;
    const size_t nr = (size_t)ni * nj * (kloc + 2);
    float *Q = (float *)calloc(nr, sizeof(float)), *S = (float *)calloc(nr, sizeof(float));
    int zstart = 1, rank = 0;
    mc_gpu_(T, &zstart, &rank);
    get_results_(Q, S, &rank);
    char msg[512];
    rc_last_error(NULL, msg, sizeof(msg));

    /* the explicit context API on the same inputs */
    rc_ctx *ctx = NULL;
    if (rc_create(&p, 0, &ctx)) return fail("rc_create");
    rc_table_set *ts2 = NULL;
    if (rc_tables_read_dir(argv[3], p.nT, p.nB, p.nQ, &ts2)) return fail("rc_tables_read_dir");
    rc_tables v;
    rc_tables_view(ts2, &v);
    if (rc_set_tables(ctx, &v)) return fail("rc_set_tables");
    rc_ticket t;
    if (rc_solve_async(ctx, T, 1, &t)) return fail("rc_solve_async");
    float *Q2 = (float *)calloc(nr, sizeof(float)), *S2 = (float *)calloc(nr, sizeof(float));
    if (rc_collect(ctx, t, Q2, S2, NULL, NULL, NULL, NULL)) return fail("rc_collect");

    int finite = 1, nonzero = 0;
    for (int k = 1; k <= kloc; ++k)
        for (int j = 1; j <= p.jmax; ++j)
            for (int i = 1; i <= p.imax; ++i) {
                const float q = Q[((size_t)k * nj + j) * ni + i];
                finite &= isfinite(q) != 0;
                nonzero |= q != 0.0f;
            }
    const int same = memcmp(Q, Q2, nr * sizeof(float)) == 0 && memcmp(S, S2, nr * sizeof(float)) == 0;
    printf("legacy_abi: %dx%dx%d photmax %d nVar %d: identical %d finite %d nonzero %d\n", p.imax, p.jmax,
           p.kmax, p.photmax, p.nVar, same, finite, nonzero);
    rc_destroy(ctx);
    rc_tables_free(ts2);
    rc_legacy_release();
    free(T);
    free(Q);
    free(S);
    free(Q2);
    free(S2);
    if (!(same && finite && nonzero)) {
        fprintf(stderr, "legacy_abi: mismatch (last library message: %s)\n", msg);
        return 1;
    }
    return 0;
}
