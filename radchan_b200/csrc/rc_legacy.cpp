// rc_legacy.cpp -- the reference's Fortran-callable entry points over one
// process-wide solver context.
//
//   mc_gpu_      (src/montecarlo/mc_gpu_noint.cu:660): copy T, launch, return
//                without waiting;
//   get_results_ (src/montecarlo/mc_gpu_noint.cu:876): wait, fill Q and the
//                Monte Carlo standard deviation in the Fortran layout;
//   rc_legacy_source (src/dns/channel.f:252-266): wait, and write the DNS's
//                Qnew, Varnew, Knew, Gnew (GET_RESULTS + fix_rad +
//                fix_kappa + the Gnew loop, rc_dns.cu).
//
// The reference configures the solver at compile time and re-reads its
// tables on every call; here the first mc_gpu_ configures the context from
// rc_legacy_configure(), or from the environment: RADCHAN_PARAM_H and
// RADCHAN_NARROWBAND_H (paths of param.h / NarrowBand.h files) and
// RADCHAN_PROPERTIES (directory of planck-mean.txt, NarrBand%d.txt,
// prob_new2.txt; default ./properties).  Errors are printed and kept for
// rc_last_error(NULL, ...); unlike the reference (cudaCheckErrors ->
// exit(1), param.h:102-112) the process is not terminated.
#include <stdio.h>
#include <stdlib.h>

#include <mutex>
#include <string>

#include "radchan.h"

namespace {
std::mutex g_mu;
rc_ctx *g_ctx = nullptr;
rc_ticket g_ticket = -1;
int g_have_ticket = 0;

void report(const char *what) {
    char buf[512];
    rc_last_error(nullptr, buf, sizeof(buf));
    fprintf(stderr, "radchan: %s failed: %s\n", what, buf);
}

// Replaces the process-wide context; the caller holds g_mu.
int configure_locked(const rc_params *p, const rc_tables *tables) {
    if (g_ctx) {
        rc_destroy(g_ctx);
        g_ctx = nullptr;
        g_have_ticket = 0;
    }
    rc_ctx *c = nullptr;
    int rc = rc_create(p, 0, &c);
    if (rc) return rc;
    if (!p->grey) {
        if (!tables) {
            rc_destroy(c);
            return RC_E_INVALID;
        }
        rc = rc_set_tables(c, tables);
        if (rc) {
            rc_destroy(c);
            return rc;
        }
    }
    g_ctx = c;
    return RC_OK;
}

// Configures the context from the environment; the caller holds g_mu.
int configure_from_env() {
    const char *ph = getenv("RADCHAN_PARAM_H");
    if (!ph) {
        fprintf(stderr, "radchan: mc_gpu_ called before rc_legacy_configure and RADCHAN_PARAM_H is not set\n");
        return RC_E_STATE;
    }
    const char *nh = getenv("RADCHAN_NARROWBAND_H");
    rc_params p;
    int rc = rc_params_from_headers(ph, nh, &p);
    if (rc) return rc;
    if (p.grey) return configure_locked(&p, nullptr);
    const char *dir = getenv("RADCHAN_PROPERTIES");
    rc_table_set *ts = nullptr;
    rc = rc_tables_read_dir(dir ? dir : "properties", p.nT, p.nB, p.nQ, &ts);
    if (rc) return rc;
    rc_tables v;
    rc_tables_view(ts, &v);
    rc = configure_locked(&p, &v);
    rc_tables_free(ts);
    return rc;
}
}  // namespace

extern "C" {

int rc_legacy_configure(const rc_params *p, const rc_tables *tables) {
    std::lock_guard<std::mutex> lk(g_mu);
    return configure_locked(p, tables);
}

int rc_legacy_release(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_ctx) rc_destroy(g_ctx);
    g_ctx = nullptr;
    g_have_ticket = 0;
    return RC_OK;
}

void mc_gpu_(float *T, int *zstart, int *rank) {
    (void)rank;
    std::lock_guard<std::mutex> lk(g_mu);
    // the first call configures the context; under the lock, so that two
    // first calls from different threads configure it once
    if (!g_ctx) {
        if (configure_from_env()) {
            report("mc_gpu_ configuration");
            return;
        }
    }
    if (g_have_ticket) {
        // a previous launch was never collected: finish it first
        rc_collect(g_ctx, g_ticket, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        g_have_ticket = 0;
    }
    int rc = rc_solve_async(g_ctx, T, zstart ? *zstart : 1, &g_ticket);
    if (rc) {
        report("mc_gpu_");
        return;
    }
    g_have_ticket = 1;
}

void get_results_(float *Q, float *sigma, int *rank) {
    (void)rank;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !g_have_ticket) {
        fprintf(stderr, "radchan: get_results_ called without a pending mc_gpu_ launch\n");
        return;
    }
    int rc = rc_collect(g_ctx, g_ticket, Q, sigma, nullptr, nullptr, nullptr, nullptr);
    g_have_ticket = 0;
    if (rc) report("get_results_");
}

int rc_legacy_source(const rc_dns_coupling *cfg, const double *T1, double *Qnew, double *Varnew, double *Knew,
                     double *Gnew, long long *n_clamped) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !g_have_ticket) {
        fprintf(stderr, "radchan: rc_legacy_source called without a pending mc_gpu_ launch\n");
        return RC_E_STATE;
    }
    int rc = rc_dns_source(g_ctx, g_ticket, cfg, T1, Qnew, Varnew, Knew, Gnew, n_clamped);
    g_have_ticket = 0;
    if (rc) report("rc_legacy_source");
    return rc;
}

}  // extern "C"
