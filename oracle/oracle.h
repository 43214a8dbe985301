/*
 * oracle.h -- CPU restatement of RadChan's OERM Monte Carlo path, used ONLY
 * as a checker (tests, the smoke check and the CPU baseline of bench.py).
 * The product never links or calls it.
 *
 * It follows src/montecarlo/mc_gpu_noint.cu (kernel_fluid :55-243,
 * march_ray :245-658, find_band :1103-1169, emiss_ang(S) :1077-1102,
 * kernel_surface :1316-1482), definitions.h:68-136 (grid) and
 * read_tables.cpp:98-220 (grey tables, wall band CDF), with the documented
 * corrections (specular y/z walls, unique Philox bundle streams, wall band
 * CDF edge rule) and the same arithmetic contract as the device code.
 */
#ifndef RADCHAN_ORACLE_H_
#define RADCHAN_ORACLE_H_
#include "radchan.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_setup {
    float Tmax, Tmin;
    int tm, row, status;
    double kappamax, Ibmax_f, Ibmax_w[2], T0, inv_dT;
} oracle_setup;

/* Full solve (or the fluid cells [cell_begin, cell_end) of the compact
 * order i fastest, then j, then local k; cell_end < 0 means all).  Outputs
 * use the compact layouts of rc_collect; entries not computed are left
 * untouched.  rpt = rays per work item of the device decomposition, which
 * fixes the FP64 summation order.  fp64 != 0 runs the full double build. */
int oracle_solve(const rc_params *p, const rc_tables *t, const float *T, int zstart, int rpt, long long cell_begin,
                 long long cell_end, int do_walls, int fp64, int nthreads, double *q64, double *var64, double *qw64,
                 double *vw64, double *steps, double *bundles);
int oracle_trace(const rc_params *p, const rc_tables *t, const float *T, int zstart, int fp64, int n,
                 const rc_bundle_id *ids, rc_trace_rec *out, int max_cells, int *cells);
int oracle_setup_scalars(const rc_params *p, const rc_tables *t, const float *T, int fp64, oracle_setup *out);
int oracle_grid_level(const rc_params *p, int level, float *xu, float *yu, float *zu, float *x, float *y, float *z);
/* cell temperatures of a multigrid level, [km][jm][im] */
int oracle_level_T(const rc_params *p, const float *T, int level, float *out);
/* particle scattering of later solves and traces (NULL: none); the arrays
 * are copied */
int oracle_set_scattering(const rc_scattering *s);

#ifdef __cplusplus
}
#endif
#endif
