/*
 * slab_abi.c -- the reference's decomposition over several GPUs, reached
 * through the legacy entry points the way the Fortran DNS reaches it: with
 * p_col ranks in param.h every rank calls mc_gpu_(T, zstart, rank) with the
 * whole field and its own first z plane (xstart(3)), and get_results_
 * returns its slab of kmax/p_col planes (src/montecarlo/mc_gpu_noint.cu:95-98
 * with num_gpu = 1 per rank; channel.f:250-256).  Here the ranks run one
 * after the other in one process on one GPU (the library's results do not
 * depend on which GPU computes a slab: bundles draw from counters of the
 * global cell index and Tmax spans the whole field).
 *
 * usage: slab_abi PARAM_H NARROWBAND_H SCRATCH_DIR   (param.h with p_col > 1)
 *
 * Exits 0 when every slab equals the same planes of the one-GPU solve of the
 * field (p_col = 1, explicit context API), bit for bit, walls included.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "radchan.h"

static int fail(const char *what) {
    char buf[512];
    rc_last_error(NULL, buf, sizeof(buf));
    fprintf(stderr, "slab_abi: %s failed: %s\n", what, buf);
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s PARAM_H NARROWBAND_H SCRATCH_DIR\n", argv[0]);
        return 2;
    }
    rc_params p;
    if (rc_params_from_headers(argv[1], argv[2], &p)) return fail("rc_params_from_headers");
    if (p.p_col < 2 || p.kmax % p.p_col) {
        fprintf(stderr, "slab_abi: param.h must set p_col > 1 dividing kmax\n");
        return 2;
    }
    /* tables in the reference's file formats; both solves read them back
     * from the files (the text format rounds the synthetic values) */
    rc_synth_spec spec = {p.nB, p.nQ, p.nT, 300.0, 2000.0, 500.0, 10000.0, -3.0, 2.0, 1.0, 1.5, 20240601u};
    rc_table_set *ts = NULL;
    if (rc_tables_synthetic(&spec, &ts)) return fail("rc_tables_synthetic");
    if (rc_tables_write_dir(ts, argv[3])) return fail("rc_tables_write_dir");
    rc_tables_free(ts);
    ts = NULL;
    if (rc_tables_read_dir(argv[3], p.nT, p.nB, p.nQ, &ts)) return fail("rc_tables_read_dir");

    const int ni = p.imax + 2, nj = p.jmax + 2, nk = p.kmax + 2;
    float *T = (float *)malloc((size_t)ni * nj * nk * sizeof(float));
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

    /* one GPU for the whole field through the context API */
    rc_params p1 = p;
    p1.p_col = 1;
    rc_ctx *ctx = NULL;
    if (rc_create(&p1, 0, &ctx)) return fail("rc_create");
    rc_tables v;
    rc_tables_view(ts, &v);
    if (rc_set_tables(ctx, &v)) return fail("rc_set_tables");
    const size_t nfull = (size_t)ni * nj * nk;
    float *Qf = (float *)calloc(nfull, sizeof(float)), *Sf = (float *)calloc(nfull, sizeof(float));
    rc_ticket t;
    if (rc_solve_async(ctx, T, 1, &t)) return fail("rc_solve_async");
    if (rc_collect(ctx, t, Qf, Sf, NULL, NULL, NULL, NULL)) return fail("rc_collect");

    /* the ranks: legacy entry points configured from the environment */
    setenv("RADCHAN_PARAM_H", argv[1], 1);
    setenv("RADCHAN_NARROWBAND_H", argv[2], 1);
    setenv("RADCHAN_PROPERTIES", argv[3], 1);
    const int kloc = p.kmax / p.p_col;
    const size_t nslab = (size_t)ni * nj * (kloc + 2);
    float *Q = (float *)calloc(nslab, sizeof(float)), *S = (float *)calloc(nslab, sizeof(float));
    int same = 1, nonzero = 0;
    for (int rank = 0; rank < p.p_col; ++rank) {
        int zstart = rank * kloc + 1, r = rank;
        mc_gpu_(T, &zstart, &r);
        get_results_(Q, S, &r);
        /* slab planes k = 1..kloc are planes zstart..zstart+kloc-1 of the field;
         * i = 0 and imax+1 hold the wall fluxes */
        for (int k = 1; k <= kloc; ++k)
            for (int j = 1; j <= p.jmax; ++j) {
                const float *a = Q + ((size_t)k * nj + j) * ni, *b = Qf + ((size_t)(zstart + k - 1) * nj + j) * ni;
                const float *c = S + ((size_t)k * nj + j) * ni, *d = Sf + ((size_t)(zstart + k - 1) * nj + j) * ni;
                same &= memcmp(a, b, ni * sizeof(float)) == 0 && memcmp(c, d, ni * sizeof(float)) == 0;
                for (int i = 1; i <= p.imax; ++i) nonzero |= a[i] != 0.0f;
            }
    }
    char msg[512];
    rc_last_error(NULL, msg, sizeof(msg));
    printf("slab_abi: %dx%dx%d in %d slabs: identical %d nonzero %d\n", p.imax, p.jmax, p.kmax, p.p_col, same,
           nonzero);
    rc_destroy(ctx);
    rc_tables_free(ts);
    rc_legacy_release();
    free(T);
    free(Q);
    free(S);
    free(Qf);
    free(Sf);
    if (!(same && nonzero)) {
        fprintf(stderr, "slab_abi: mismatch (last library message: %s)\n", msg);
        return 1;
    }
    return 0;
}
