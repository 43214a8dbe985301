/*
 * radchan.h -- C ABI of the B200 (sm_100a) narrow-band correlated-k OERM
 * Monte Carlo radiative-transfer solver.
 *
 * This library is a drop-in for the GPU radiation solver of RadChan
 * (src/montecarlo).  The reference exposes two Fortran-callable symbols,
 * declared here with the same names, arguments and array layouts:
 *
 *   mc_gpu_      (src/montecarlo/mc_gpu_noint.cu:660)  -- launch, returns
 *                without waiting for the device;
 *   get_results_ (src/montecarlo/mc_gpu_noint.cu:876)  -- wait, fill Q and
 *                its Monte Carlo standard deviation.
 *
 * The reference configures everything at compile time (src/param/param.h,
 * src/param/NarrowBand.h) and reads its spectral tables from
 * the text files in properties/ on every call (src/montecarlo/read_tables.cpp:21-96).
 * Here the same parameter set is a runtime struct (rc_params), which can be
 * filled from an existing param.h / NarrowBand.h pair, and the tables are
 * uploaded once and stay resident on the device.
 *
 * Conventions
 *  - Every rc_* function returns an int status: RC_OK (0) or a negative
 *    RC_E* code; rc_last_error() returns the message of the last failure
 *    on that context (or of the last context-free call when ctx is NULL).
 *  - All buffers passed in belong to the caller; the library copies them.
 *  - Temperature fields are float, Fortran order (i fastest), with one
 *    ghost layer: T(0:imax+1, 0:jmax+1, 0:kmax+1), index
 *    i + (imax+2)*(j + (jmax+2)*k)   (param.h:132 idx_T).
 *  - Result arrays are float Q(0:imax+1, 0:jmax+1, 0:kloc+1) with
 *    kloc = kmax/p_col (param.h:138 idx_F, mc_gpu_noint.cu:876): interior
 *    cells receive the radiative source (W/m^3 with SI tables), i = 0 and
 *    i = imax+1 receive the net wall flux (W/m^2) of adiabatic x-walls when
 *    calcwalls = 1, else 0.  Other ghost entries are left untouched.
 *  - One context per host thread; a context is not re-entrant.  The
 *    library never calls cudaDeviceReset.
 */
#ifndef RADCHAN_H_
#define RADCHAN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RC_MAX_LEVELS 9   /* param.h:24 grid_num is at most 9 */

/* status codes */
#define RC_OK            0
#define RC_E_INVALID    -1   /* bad argument or parameter combination */
#define RC_E_CUDA       -2   /* a CUDA runtime call failed */
#define RC_E_NOMEM      -3   /* device or host allocation failed / budget */
#define RC_E_IO         -4   /* table file missing or malformed */
#define RC_E_STATE      -5   /* call out of order (e.g. collect w/o solve) */
#define RC_E_RANGE      -6   /* T outside the table range or not finite */
#define RC_E_BUSY       -7   /* no free slot / queue full */
#define RC_E_NOTFOUND   -8
#define RC_E_CANCELLED  -9   /* a served request was cancelled */
#define RC_E_TIMEOUT   -10   /* a multi-GPU group did not form or a collective did not finish in time */

/* wall indices: west (x=0), east (x=Lx), south (y=0), north (y=Ly),
 * bottom (z=0), top (z=Lz) -- the order of param.h:68-100 */
enum { RC_WEST = 0, RC_EAST, RC_SOUTH, RC_NORTH, RC_BOT, RC_TOP };

/* boundary types, param.h:90-94 */
#define RC_BD_PERIODIC 1
#define RC_BD_BLACK    2
#define RC_BD_SPECULAR 3
#define RC_BD_ADIABLK  4   /* black wall at the temperature of the first cell */
#define RC_BD_LOST     5

/* Runtime image of src/param/param.h + NarrowBand.h. */
typedef struct rc_params {
    int imax, jmax, kmax;               /* param.h:10-12 */
    float Lx, Ly, Lz;                   /* param.h:13-15 (m) */
    double fact_mesh;                   /* param.h:16 parabolic x stretching */
    int nVar;                           /* param.h:18 replicates */
    int photmax;                        /* param.h:19 bundles per cell and replicate */
    double chanHeight;                  /* param.h:20 scales k and kP on load */
    int grid_num;                       /* param.h:24 */
    int maxi[RC_MAX_LEVELS], maxj[RC_MAX_LEVELS], maxk[RC_MAX_LEVELS]; /* :27-29 */
    int maxs[RC_MAX_LEVELS];            /* param.h:31-49 step budget per level */
    int num_gpu, p_col;                 /* param.h:8-9 (num_gpu must be 1) */
    int num_streams, blockdim, nblocks; /* param.h:52-54, accepted as hints */
    int srt;                            /* param.h:57 band-sorted bundle order */
    int grey;                           /* param.h:59 grey gas (NarrowBand.h:213-221) */
    int calcwalls;                      /* param.h:61 wall-flux kernel */
    int random;                         /* param.h:63 (Sobol in the reference; here
                                           Philox counters are always used) */
    int floatpoint;                     /* param.h:65 1 -> full FP64 kernels */
    float eps[6];                       /* param.h:68-73 wall emissivities */
    float Tw[6];                        /* param.h:75-80 wall temperatures (K) */
    int adiabw, adiabe;                 /* param.h:82-83 */
    double stefan;                      /* param.h:85 */
    float toll, tollS;                  /* param.h:86-87 transmissivity cutoffs */
    int bd[6];                          /* param.h:95-100 */
    /* grey-gas constants, NarrowBand.h:214-219 */
    int grey_nT, grey_nB;
    float abscoeff, Tmins, wvmax;
    /* narrow-band table dimensions, NarrowBand.h:189-191 */
    int nT, nQ, nB;
    /* Philox key of the bundle streams */
    uint64_t seed;
} rc_params;

/* Spectral tables in the reference's layout (read_tables.cpp:21-96).
 * kq and kP are given unscaled; the library multiplies them by
 * chanHeight as readT does (read_tables.cpp:30,56). */
typedef struct rc_tables {
    int nT, nB, nQ;
    const float *Tnb;    /* [nT] table temperatures, uniformly spaced (K) */
    const float *kP;     /* [nT] Planck-mean absorption coefficient */
    const float *wvl;    /* [nB] band left edge (cm^-1) */
    const float *wvr;    /* [nB] band right edge (cm^-1) */
    const float *wvc;    /* [nB] band centre (cm^-1) */
    const float *kavg;   /* [nB] band-mean k used as the sort key (srt) */
    const float *kq;     /* [nB][nT][nQ] k at each g point */
    const float *prob;   /* [nT][nB] cumulative band probability */
    const float *probg;  /* [nT][nB][nQ] cumulative g probability */
    const float *wq;     /* [nQ] g-quadrature weights */
} rc_tables;

/* Seeded synthetic correlated-k table recipe: k_{b,g}(T) =
 * k0_b exp(kexp xi_g) (T/1000)^{n_b}, log10 k0_b ~ U[logk_lo, logk_hi],
 * n_b ~ U[-nexp, nexp], xi_g the nQ-point Gauss-Legendre nodes on [-1,1],
 * band centres ~ U[nu_lo, nu_hi] sorted, nT temperatures on [T_lo, T_hi]. */
typedef struct rc_synth_spec {
    int nB, nQ, nT;
    double T_lo, T_hi;
    double nu_lo, nu_hi;
    double logk_lo, logk_hi;
    double nexp, kexp;
    uint64_t seed;
} rc_synth_spec;

/* Host-owned table set (returned by the builders below). */
typedef struct rc_table_set rc_table_set;

typedef struct rc_ctx rc_ctx;
typedef int32_t rc_ticket;

/* ---------------- parameters ---------------- */

/* Fill with the reference's defaults (param.h, NarrowBand.h as shipped). */
int rc_params_default(rc_params *p);
/* Parse an existing param.h and (optional) NarrowBand.h: #define lines,
 * the maxi/maxj/maxk/maxs initialisers and their #if grid_num branches. */
int rc_params_from_headers(const char *param_h, const char *narrowband_h, rc_params *p);
/* Check a parameter set; returns RC_E_INVALID with a message on failure. */
int rc_params_validate(const rc_params *p, char *msg, size_t msglen);

/* ---------------- tables ---------------- */

int rc_tables_synthetic(const rc_synth_spec *spec, rc_table_set **out);
/* Read properties/planck-mean.txt, NarrBand%d.txt and prob_new2.txt from
 * dir in the formats of nbcorrk/write_tables.cpp:23-107. */
int rc_tables_read_dir(const char *dir, int nT, int nB, int nQ, rc_table_set **out);
int rc_tables_write_dir(const rc_table_set *ts, const char *dir);
/* Check what the solver assumes of a table set (rc_set_tables runs the same
 * check): 2..256 increasing, uniformly spaced temperatures; cumulative
 * probabilities finite, non-decreasing and within [0, 1]; absorption and
 * Planck-mean coefficients finite and >= 0.  RC_E_INVALID with the first
 * violation in msg otherwise.  Needs no GPU. */
int rc_tables_validate(const rc_tables *t, char *msg, size_t msglen);
/* Borrowed view of a table set (valid until rc_tables_free). */
int rc_tables_view(const rc_table_set *ts, rc_tables *view);
void rc_tables_free(rc_table_set *ts);

/* ---------------- scattering particles ---------------- */

/* Scattering by suspended particles.  The reference's Monte Carlo path has
 * no scattering; its table generator tabulates the particles: per band the
 * absorption and scattering coefficients at each g point
 * (nbcorrk/write_tables.cpp:204-260, writeP) and the cumulative
 * phase-function probability over the scattering angle
 * (nbcorrk/write_tables.cpp:326-336, writeH, built by
 * nbcorrk/calc_prob.cpp:253-270).  Absorption by the particles belongs in
 * the absorption tables (rc_tables); this adds their scattering.  Bands and
 * g points are the context's (grey gas: grey_nB bands, nQ = 1). */
typedef struct rc_scattering {
    int nB, nQ, nA;
    const float *ksca;       /* [nB][nQ] scattering coefficient (1/m; scaled by
                                chanHeight on upload like k); no temperature axis */
    const float *kabs;       /* [nB][nQ] particle absorption from the files, or
                                NULL; informational (fold it into rc_tables) */
    const float *theta;      /* [nA] scattering angles (radians), increasing from 0,
                                at most pi */
    const float *phase_cdf;  /* [nB][nA] cumulative probability of the scattering
                                angle: 0 at theta[0], non-decreasing, 1 at theta[nA-1] */
} rc_scattering;

/* Seeded synthetic particle tables: Henyey-Greenstein phase function
 * p(cos t) = (1 - g^2) / (1 + g^2 - 2 g cos t)^(3/2) per band with asymmetry
 * g_b ~ U[g_lo, g_hi], tabulated at nA angles j pi / (nA - 1) and integrated
 * as calc_prob.cpp:253-270 does (trapezoids of p sin t, normalised by the
 * last); ksca_b ~ log-uniform on [ksca_lo, ksca_hi], the same at every g
 * point; kabs 0. */
typedef struct rc_scatter_spec {
    int nB, nQ, nA;
    double ksca_lo, ksca_hi;
    double g_lo, g_hi;
    uint64_t seed;
} rc_scatter_spec;

/* Host-owned particle table set. */
typedef struct rc_scatter_set rc_scatter_set;

int rc_scattering_synthetic(const rc_scatter_spec *spec, rc_scatter_set **out);
/* Read dir/NarrBand%d.txt (writeP format: "wvl wvr wvc", then the nQ
 * absorption and the nQ scattering coefficients) for nB bands and
 * dir/prob_scatt.txt (writeH format: "theta wvc cdf" for every band and
 * angle, angles fastest; nA is the row count over nB). */
int rc_scattering_read_dir(const char *dir, int nB, int nQ, rc_scatter_set **out);
int rc_scattering_write_dir(const rc_scatter_set *s, const char *dir);
/* What the march assumes of particle tables: 1 <= nB, nQ; 2 <= nA <= 4096;
 * ksca finite and >= 0; angles finite, strictly increasing, theta[0] >= 0,
 * theta[nA-1] <= pi; every band's CDF finite, non-decreasing, 0 at the
 * first angle and within 1e-6 of 1 at the last.  RC_E_INVALID with the
 * first violation in msg otherwise.  Needs no GPU. */
int rc_scattering_validate(const rc_scattering *s, char *msg, size_t msglen);
/* Borrowed view (valid until rc_scattering_free). */
int rc_scattering_view(const rc_scatter_set *s, rc_scattering *view);
void rc_scattering_free(rc_scatter_set *s);

/* ---------------- solver context ---------------- */

int rc_create(const rc_params *p, int device, rc_ctx **out);
int rc_set_tables(rc_ctx *ctx, const rc_tables *t);
/* Particle scattering for the context's later solves (NULL removes it; no
 * counterpart in the reference, whose medium only absorbs and emits).
 * Bundles then travel a free path drawn against the scattering coefficient
 * of their band and g point, turn by an angle drawn from the band's phase
 * function and a uniform azimuth at each event, and keep absorbing along
 * the way as before; every draw comes from the bundle's own Philox counter
 * (emission's, with an event number), so results stay independent of the
 * launch shape.  Batches run such contexts in the scattering variant of the
 * march; the server takes particles per table set
 * (rc_server_set_scattering).  Set it between solves (no solve of the
 * context in flight). */
int rc_set_scattering(rc_ctx *ctx, const rc_scattering *s);
/* Copy T (host, whole field incl. ghosts) and launch; returns at once. */
int rc_solve_async(rc_ctx *ctx, const float *T, int zstart, rc_ticket *ticket);
/* Same with T already in device memory (same layout). */
int rc_solve_device_async(rc_ctx *ctx, const float *T_dev, int zstart, rc_ticket *ticket);
/* Wait for a ticket and fill the caller's arrays.  Q and sigma use the
 * Fortran result layout above (either may be NULL).  The optional double
 * outputs use compact layouts: q64/var64 [kloc][jmax][imax] (per-cell mean
 * and variance of the mean), qw64/vw64 [2][kloc][jmax] (west, east). */
int rc_collect(rc_ctx *ctx, rc_ticket ticket, float *Q, float *sigma,
               double *q64, double *var64, double *qw64, double *vw64);
/* Wait for a ticket and copy its compact double results (layouts as in
 * rc_collect) into the caller's device arrays (any may be NULL); the
 * ticket is consumed.  For callers that gather results over NCCL. */
int rc_collect_device(rc_ctx *ctx, rc_ticket ticket, double *q64_dev, double *var64_dev,
                      double *qw64_dev, double *vw64_dev);
/* Device-side results of the last collected/finished ticket (no copy):
 * pointers to the compact double arrays described above. */
int rc_device_results(rc_ctx *ctx, rc_ticket ticket, const double **q64,
                      const double **var64, const double **qw64, const double **vw64);
/* Per-solve diagnostics of a finished ticket. */
typedef struct rc_solve_info {
    float Tmax;            /* max of interior T and x-wall face averages */
    float kappamax;        /* Planck-mean k at Tmax */
    float Ibmax_fluid;     /* energy per fluid bundle */
    int   table_row;       /* table row nearest Tmax (mc_gpu_noint.cu:1110) */
    int   status;          /* bit 0: T outside table range, bit 1: non-finite T;
                              bounds-checked build (libradchan_checked.so): bit 3 an
                              index was out of bounds, bits 8-15 the first such site */
    double bundles;        /* bundles traced */
    double steps;          /* ray-cell steps */
    float ms_device;       /* device time of the march kernel */
    float ms_solve;        /* device time of the whole solve (copy-in .. tally) */
} rc_solve_info;
int rc_solve_info_get(rc_ctx *ctx, rc_ticket ticket, rc_solve_info *info);
/* Launch knobs of the march kernel; values <= 0 (sort_bands < 0) keep the
 * current setting.  rays_per_thread: bundles per work item (power of two
 * <= 64; it fixes the FP64 summation grouping, results differ only by
 * rounding); block_threads: 128 or 256; sort_bands: 1 hands each warp's
 * emitted bundles to its lanes in ascending absorption coefficient, so rays
 * traced side by side have similar path lengths (the execution-order part
 * of the reference's srt band sorting, mc_gpu_noint.cu:1270-1294);
 * occupancy: resident 256-thread blocks per SM the register budget must
 * allow (2, 3 or 4).  None of them changes which bundles are traced. */
int rc_set_launch(rc_ctx *ctx, int rays_per_thread, int block_threads, int sort_bands, int occupancy);
int rc_get_launch(rc_ctx *ctx, int *rays_per_thread, int *block_threads, int *sort_bands, int *occupancy);
/* Long-ray priority of rc_solve_async / rc_solve_device_async.  A bundle
 * whose path is long -- nearly parallel to the x walls, so that it crosses
 * the periodic y/z boundaries again and again, and in a near-transparent
 * band and g point -- takes up to the last level's step budget, and when it
 * starts late in a launch the GPU waits for it alone.  Before the march a
 * short pass draws every bundle's direction, band and g point exactly as
 * emission will, estimates its path length as min(d_x / |s_x|,
 * ln(1/tol) / k_min) (d_x the distance to the x wall it heads for, k_min the
 * smallest k of its band and g point over the table rows the field spans)
 * and lists the tiles holding a bundle whose estimate exceeds `threshold`
 * channel widths Lx; the march claims those tiles first.  Default
 * RC_PRIORITY_DEFAULT; 0 turns it off.  It changes the order of the work,
 * never a result.  Each solve slot builds the list on its first solve and
 * reuses it while the draws and the work decomposition stay the same (seed,
 * photmax, rays_per_thread, replicates, grid, walls, threshold): a later
 * field can only make the order less apt.  Solves of more than 2^22 tiles
 * skip it (there, reordering cost more than the tail it removed). */
#define RC_PRIORITY_DEFAULT 12.0f
int rc_set_priority(rc_ctx *ctx, float threshold);
/* Try launch configurations on T (host) with a reduced bundle count
 * (pilot_photmax, raised until a pilot launch has 10^8 bundles, at most the
 * context's photmax; <= 0: the context's photmax) and keep the fastest:
 * rays_per_thread x block_threads x occupancy with sorting off, then
 * sort_bands on at the best of those.  Each configuration is scored by the
 * estimated time of the real solve: its pilot march time (best of two
 * launches after a warm-up) scaled to the context's photmax -- when that is
 * more than 4x the pilot, from the pilot timed at one and at two times its
 * photmax, so the marginal cost per bundle carries the estimate and not the
 * pilot's tail -- plus writing and reading the FP64 partial sums that
 * rays_per_thread implies at that photmax.  The current knobs are the
 * incumbent, and another configuration must beat them by 3 %.  Writes the
 * chosen knobs. */
int rc_autotune(rc_ctx *ctx, const float *T, int zstart, int pilot_photmax,
                int *rays_per_thread, int *block_threads, int *sort_bands, int *occupancy);
/* Solve without allocating device memory (this entry point has no
 * counterpart in the reference).  For callers that cannot call cudaMalloc
 * while they run -- a time-stepping code whose device memory is owned by
 * another allocator or reserved up front, or that must not add allocation
 * latency or failure points to a step -- this runs the same kernels as
 * rc_solve_device_async, but the march's partial sums go to a
 * library-owned static device array of 64 MiB (8,388,608 doubles: one per
 * cell x replicate x part of the photmax/rays_per_thread decomposition,
 * plus the wall cells) instead of a buffer the library would allocate.
 * Sizes beyond that return RC_E_INVALID.  T_dev is the whole field in
 * device memory; q64/var64 (required) and qw64/vw64 (optional) are the
 * caller's device arrays in the compact layouts of rc_collect.  The call
 * returns when the results are written.  The array is set up on the first
 * call on each device (make that first call before any stream capture) and
 * keeps its contents between calls; every element a solve reads is written
 * by the same solve first.  All calls in the process share the one array,
 * so calls that overlap on the GPU (several contexts or threads) race.
 * qw64/vw64 rows of a wall whose flux is not computed are set to 0.  With
 * no ticket to read rc_solve_info from, the solve's status word is reported
 * by the return code: RC_E_RANGE, with the outputs written, when T was not
 * finite (status bit 1), an index was out of bounds (bit 3, bounds-checked
 * build; the message names the site) or T lay outside the table range
 * (bit 0, end rows used); rc_last_error says which. */
int rc_solve_noalloc(rc_ctx *ctx, const float *T_dev, int zstart, double *q64_dev, double *var64_dev,
                     double *qw64_dev, double *vw64_dev);
int rc_destroy(rc_ctx *ctx);
/* The parameters a context was created with and its device (either output
 * may be NULL). */
int rc_get_params(const rc_ctx *ctx, rc_params *p, int *device);
int rc_last_error(const rc_ctx *ctx, char *buf, size_t len);
/* Failure injection for tests of the error paths (no counterpart in the
 * reference): the next `count` times the named host-side site is reached
 * (in any context or server of the process) it fails with RC_E_CUDA and
 * the message "injected failure at <site>", without making its CUDA call,
 * so no device fault is involved.  count 0 disarms.  Sites: "field_copy"
 * (a solve's field copy and set-up), "march" and "tally" (their launches),
 * "collect" (result copies), "dns" (the DNS coupling launch), "quantum"
 * (a server march launch). */
int rc_debug_fail_next(const char *site, int count);
/* Grid faces/centres of level `level` as built by the library
 * (definitions.h:68-136); any pointer may be NULL. */
int rc_grid_level(const rc_params *p, int level, float *xu, float *yu, float *zu,
                  float *x, float *y, float *z);

/* ---------------- bundle traces (parity checks) ---------------- */

/* One traced bundle: kind 0 = fluid cell (i,j,k), 1 = west wall (j,k),
 * 2 = east wall (j,k); v replicate; h bundle index. */
typedef struct rc_bundle_id { int kind, i, j, k, v, h; } rc_bundle_id;
typedef struct rc_trace_rec {
    int nb, g;             /* sampled band and g point */
    int nsteps;            /* ray-cell steps taken */
    int end_level;         /* multigrid level at the end */
    float sx, sy, sz;      /* emission direction */
    float tra;             /* final transmissivity */
    double De;             /* the bundle's tally contribution */
} rc_trace_rec;
/* Trace bundles of the ticket's problem; cells[n*max_cells*4] receives
 * (level, ic, jc, kc) of the first max_cells steps of each bundle. */
int rc_trace(rc_ctx *ctx, rc_ticket ticket, int n, const rc_bundle_id *ids,
             rc_trace_rec *out, int max_cells, int *cells);
/* Band and g point that emission of the ticket's solve selects for
 * caller-given uniforms u_band[n], u_g[n] (no counterpart in the reference;
 * it exposes find_band / find_bandS, mc_gpu_noint.cu:1103-1233, for checks
 * of their edge rules: u < cdf[0] -> 0, u == 1 -> last).  kind 0 searches
 * the fluid band CDF at the table row nearest Tmax and the g CDF of that
 * band, kind 1 or 2 the wall band CDF and the g weights' CDF. */
int rc_sample_bands(rc_ctx *ctx, rc_ticket ticket, int kind, int n, const float *u_band,
                    const float *u_g, int *nb, int *g);

/* ---------------- diagnostics ---------------- */

/* Random-sector gather throughput of this GPU (no counterpart in the
 * reference): every lane reads 4 bytes from a pseudo-random 32-byte sector
 * of a device array of `bytes` bytes, eight independent reads in flight,
 * at full occupancy; mode 0 reads through L2 only (ld.global.cg), mode 1
 * through the read-only L1 path as the march does.  *sectors_per_s is the
 * best of three timed launches after a warm-up launch (CUDA events);
 * *ms_best (optional) that launch's time.  With `bytes` at the size of a
 * solve's temperature pyramid and tables it is the ceiling of the march's
 * gathers, which stay L2-resident. */
int rc_probe_gather(int device, size_t bytes, int mode, int iters, double *sectors_per_s, float *ms_best);

/* ---------------- one solve over several GPUs (NCCL) ---------------- */

/* The reference spreads one solve over GPUs and nodes by z slabs of the
 * emitting cells while every GPU holds the whole field (mc_gpu_noint.cu:
 * 95-98: kloc = kmax/p_col planes from zstart), and the DNS combines the
 * slabs' results over MPI (fixvar.f:202-203).  These calls do the same from
 * C over NCCL, one process (or thread) per GPU: rank r of a group of N
 * solves the planes rc_slab_range names, of the field that rank 0 holds,
 * and every rank ends with the whole solution.  Bundles draw from counters
 * of the global cell index, so the gathered solution equals the one-GPU
 * solve of the same problem bit for bit.  NCCL is loaded when the first id
 * or communicator is made (libnccl.so.2, or the file RC_NCCL_LIBRARY
 * names); the rest of the library does not need it.  There is no other
 * data-path collective: the field is broadcast once and the results are
 * all-gathered once per solve. */
#define RC_SLAB_ID_BYTES 128   /* NCCL_UNIQUE_ID_BYTES */
typedef struct rc_slab_comm rc_slab_comm;
/* Planes of rank `rank` in a group of `nranks`: kloc = kmax/nranks planes
 * starting at the 1-based zstart = rank*kloc + 1 (kmax must be a multiple
 * of nranks, as p_col requires in the reference). */
int rc_slab_range(int kmax, int nranks, int rank, int *kloc, int *zstart);
/* A new group id, made on one rank; every rank passes the same
 * RC_SLAB_ID_BYTES bytes to rc_slab_comm_create (e.g. after MPI_Bcast). */
int rc_slab_unique_id(void *id);
/* Joins group `id` as rank `rank` of `nranks` on `device`.  Returns once
 * every rank has joined; after timeout_s seconds (<= 0: 300) without that,
 * RC_E_TIMEOUT and the group is abandoned.  The same timeout bounds every
 * later collective of the communicator: one that does not finish in time
 * aborts the group (RC_E_TIMEOUT; the communicator is then unusable and
 * only rc_slab_comm_destroy is valid). */
int rc_slab_comm_create(int device, int nranks, int rank, const void *id, double timeout_s,
                        rc_slab_comm **out);
/* One solve of ctx's problem over the group.  Every rank calls it with a
 * context of the same problem created with p_col = nranks on the
 * communicator's device (tables and launch knobs set alike).  T: the whole
 * field (kmax+2, jmax+2, imax+2) on every rank; rank 0's is broadcast into
 * the others' (their contents are overwritten).  q64/var64
 * [kmax][jmax][imax] (required) and qw64/vw64 [2][kmax][jmax] (optional)
 * receive the whole solution in the compact layouts of rc_collect on every
 * rank.  Each array may be device memory of the communicator's GPU (used
 * in place) or host memory (staged through device buffers the communicator
 * keeps); device memory of another GPU is refused (RC_E_INVALID).  Returns when
 * the results are in place.  A solve error on one rank (RC_E_RANGE for a
 * non-finite field, which every rank sees) is returned after the
 * collectives, so the ranks stay in step; an argument error is returned
 * before them, and the other ranks' collectives then end by the timeout. */
int rc_slab_solve(rc_slab_comm *comm, rc_ctx *ctx, float *T, double *q64, double *var64, double *qw64,
                  double *vw64);
/* Message of the communicator's last failure. */
int rc_slab_last_error(const rc_slab_comm *comm, char *buf, size_t len);
/* Leaves the group (collective over the ranks of a healthy group; a group
 * that timed out is aborted instead) and frees the communicator. */
int rc_slab_comm_destroy(rc_slab_comm *comm);

/* ---------------- batched solves ---------------- */

typedef struct rc_batch rc_batch;
/* A batch runs many contexts' solves (uneven grids, tables, photmax) in
 * one persistent work-queue launch; with use_graph the whole sequence
 * (copies + kernels) is captured once and replayed.  The members' fields
 * are copied by one kernel, their set-up kernels run as parallel chains,
 * and the march takes the tiles in natural order.  Every run also gathers
 * the members' float results (Q, sigma, wall fluxes) into one buffer
 * copied to the host once, so rc_batch_collect with only Q / sigma copies
 * nothing more. */
int rc_batch_create(int device, int use_graph, rc_batch **out);
int rc_batch_add(rc_batch *b, rc_ctx *ctx, const float *T_host, int zstart);
int rc_batch_run(rc_batch *b);          /* enqueue (after the previous run of the batch has finished); returns at once */
int rc_batch_wait(rc_batch *b, float *ms_device);
/* Device time of the last run by phase: set-up of every member (field
 * copies, set-up kernels), the march, and tally plus result copies.  Waits
 * for the run. */
int rc_batch_phases(rc_batch *b, float *ms_setup, float *ms_march, float *ms_tally);
int rc_batch_collect(rc_batch *b, int index, float *Q, float *sigma,
                     double *q64, double *var64, double *qw64, double *vw64);
int rc_batch_destroy(rc_batch *b);

/* ---------------- serving ---------------- */

typedef struct rc_server rc_server;
typedef struct rc_request {
    const rc_params *params;     /* grid, photmax (0 -> from tolerance), ... */
    int table_set;               /* id from rc_server_add_tables */
    const float *T;              /* host field, copied at submit */
    int zstart;
    float tolerance;             /* target rel. std of max|Q| (0: use photmax) */
} rc_request;
typedef struct rc_result_info {
    double t_submit, t_admit, t_done;   /* seconds, server clock */
    int photmax;                        /* bundles per cell used */
    float rel_std_maxq;                 /* RMS sigma of the cells with |Q| >= 0.9 max|Q|, over max|Q| */
    int status;
} rc_result_info;
int rc_server_create(int device, double hbm_budget_bytes, int max_inflight, rc_server **out);
int rc_server_add_tables(rc_server *s, const rc_tables *t, int *table_set);
/* Particle scattering for the requests of a table set (table_set -1: grey
 * requests; NULL removes it), copied.  Requests submitted afterwards solve
 * in that medium; a request keeps the particles current when it was
 * submitted, and contexts are pooled per table set and particle set. */
int rc_server_set_scattering(rc_server *s, int table_set, const rc_scattering *sc);
int rc_server_submit(rc_server *s, const rc_request *req, int64_t *id);
/* Wait for a request; Q/sigma in the Fortran result layout (may be NULL). */
int rc_server_wait(rc_server *s, int64_t id, float *Q, float *sigma, rc_result_info *info);
int rc_server_stats(rc_server *s, double *solves, double *busy_s, double *hbm_in_use);
/* Tiles (32 work items each) per march launch, shared among the running
 * requests: smaller quanta let new requests start sooner, larger ones cost
 * fewer launches.  0 (the default) sizes each quantum from the backlog: a
 * 32nd of the running requests' remaining tiles, between 131072 and
 * 524288. */
int rc_server_set_quantum(rc_server *s, long long tiles);
/* March launches issued so far. */
int rc_server_quanta(rc_server *s, long long *quanta);
/* How a quantum's tiles are shared among the running requests:
 * RC_SCHED_SRPT (default) serves the requests with the least remaining
 * work first, above a floor of 1/8 of the quantum shared by all;
 * RC_SCHED_FAIR gives every request an equal share. */
#define RC_SCHED_FAIR 0
#define RC_SCHED_SRPT 1
int rc_server_set_policy(rc_server *s, int policy);
/* Cancel a request: a queued one is dropped at once; a running one stops
 * after the quanta in flight finish and its context returns to the pool.
 * rc_server_wait then returns RC_E_CANCELLED (or the result, if the solve
 * completed first).  RC_E_STATE if its result is already published,
 * RC_E_NOTFOUND for an unknown (or already waited) id. */
int rc_server_cancel(rc_server *s, int64_t id);
int rc_server_destroy(rc_server *s);

/* ---------------- DNS coupling ---------------- */

/* What the channel DNS does with a finished solve before its energy
 * equation uses it (src/dns/channel.f:249-266): GET_RESULTS, then fix_rad
 * (fixvar.f:179-242: Q and sigma over stefan Tin^4, wall fluxes also over
 * Height, the DNS rank's j pencil cut out), fix_kappa (fixvar.f:16-43:
 * Planck-mean coefficient at T1 Tin by linear_int), then
 * Qnew *= underrelax and Gnew = 4 T1^4 - Qnew / Knew. */
#define RC_DNS_MAX_T 128
typedef struct rc_dns_coupling {
    double Tin;          /* temperature scale, K: T = T1 Tin (channel.f:111) */
    double Height;       /* divides the wall fluxes (fixvar.f:223-224; channel.f:106) */
    double underrelax;   /* multiplies Qnew before Gnew is formed (channel.f:263) */
    double stefan;       /* Stefan-Boltzmann constant of the DNS (param.txt:41: 5.67e-08) */
    int nTemp;           /* rows of Tnb and kP, 2..RC_DNS_MAX_T */
    const double *Tnb;   /* [nTemp] table temperatures, K, ascending with a uniform step >= 1 K */
    const double *kP;    /* [nTemp] Planck-mean coefficient already times Height (read_kP, fixvar.f:1-14) */
    int jstart, jend;    /* 1-based global j range of the DNS pencil (xstart(2), xend(2)) */
} rc_dns_coupling;
/* Wait for a ticket and write the DNS source terms of the pencil
 * j = jstart..jend (jn = jend - jstart + 1), k = 1..kloc of the solve:
 *   Qnew   = Q / stefan / Tin^4 (walls i = 0, imax+1: then / Height), x underrelax
 *   Varnew = sigma / stefan / Tin^4
 *   Knew   = kP at T1 Tin, row t = int(T1 Tin - Tnb[0]) / int(Tnb[1] - Tnb[0])
 *            (the truncating rule of linear_int, fixvar.f:35-43)
 *   Gnew   = 4 T1^4 - Qnew / Knew   (T1^4 evaluated as (T1 T1)(T1 T1))
 * with Q and sigma exactly the values rc_collect / get_results_ give.
 * T1 is the DNS's nondimensional temperature pencil (0:imax+1, 0:jn+1,
 * 0:kloc+1), i fastest; the four outputs are (0:imax+1, jn, kloc) doubles.
 * Where the row falls outside 0..nTemp-2 (the reference reads past its table
 * there) the end interval is extended and the cell is counted in
 * *n_clamped (optional).  The ticket is consumed, as by rc_collect. */
int rc_dns_source(rc_ctx *ctx, rc_ticket ticket, const rc_dns_coupling *cfg, const double *T1,
                  double *Qnew, double *Varnew, double *Knew, double *Gnew, long long *n_clamped);
/* The same on device arrays, enqueued on `stream` (a cudaStream_t; NULL:
 * the solve's own stream -- the legacy default stream cannot be named)
 * behind the solve; returns at once.  The ticket
 * stays valid (collect or release it afterwards) and the next solve in its
 * slot waits for this kernel.  n_clamped_dev (optional) is a device
 * counter that the kernel adds to. */
int rc_dns_source_device(rc_ctx *ctx, rc_ticket ticket, const rc_dns_coupling *cfg, const double *T1_dev,
                         double *Qnew_dev, double *Varnew_dev, double *Knew_dev, double *Gnew_dev,
                         unsigned long long *n_clamped_dev, void *stream);

/* ---------------- reference-compatible entry points ---------------- */

/* Configure the process-wide context used by mc_gpu_/get_results_.
 * tables may be NULL in grey mode.  Without this call the first mc_gpu_
 * reads RADCHAN_PARAM_H / RADCHAN_NARROWBAND_H (paths of the reference's
 * headers) and RADCHAN_PROPERTIES (directory of the table files, default
 * ./properties). */
int rc_legacy_configure(const rc_params *p, const rc_tables *tables);
int rc_legacy_release(void);
/* mc_gpu_noint.cu:660 -- T is the whole (0:imax+1,0:jmax+1,0:kmax+1) field,
 * zstart the 1-based first z index of this slab; returns before the device
 * finishes.  Errors are printed and kept for rc_last_error(NULL, ...). */
void mc_gpu_(float *T, int *zstart, int *rank);
/* mc_gpu_noint.cu:876 -- waits, then fills Q and sigma (Fortran layout). */
void get_results_(float *Q, float *sigma, int *rank);
/* channel.f:252-266 in one call: waits for the pending mc_gpu_ launch and
 * writes the DNS source terms as rc_dns_source does (replaces GET_RESULTS,
 * fix_rad, fix_kappa and the Gnew loop). */
int rc_legacy_source(const rc_dns_coupling *cfg, const double *T1, double *Qnew, double *Varnew,
                     double *Knew, double *Gnew, long long *n_clamped);

#ifdef __cplusplus
}
#endif
#endif /* RADCHAN_H_ */
