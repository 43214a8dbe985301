// oracle.cpp -- CPU restatement of RadChan's OERM Monte Carlo radiative
// source (src/montecarlo).  TEST INFRASTRUCTURE ONLY: tests, the smoke
// check and bench.py's CPU baseline use it as the checker; the product
// (radchan_b200/libradchan.so) never links it.
//
// Structure follows the reference: per cell, per replicate, per bundle
// (kernel_fluid, mc_gpu_noint.cu:92-239), a march that loops over the
// multigrid levels with a while loop per level (march_ray :245-658 called
// from :210-224), band/g bisection (find_band :1103-1169), and the wall
// kernel (kernel_surface :1316-1482).  Arithmetic follows the contract
// written at the top of radchan_b200/csrc/rc_device.cuh so that bundle
// draws, traversals and tallies can be compared bit for bit.
#include "oracle.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "radchan_math.h"

namespace {

template <typename R> struct M;
template <> struct M<float> {
    static float expm1_(float x) { return rc_expm1f(x); }
    static float log_(float x) { return rc_logf(x); }
    static float sqrt_(float x) { return sqrtf(x); }
    static void sincos2pi_(float u, float *s, float *c) { rc_sincos2pif(u, s, c); }
    static float fma_(float a, float b, float c) { return fmaf(a, b, c); }
    static float lerp_(float a0, float a1, float w) { return rc_lerpf(a0, a1, w); }
};
template <> struct M<double> {
    static double expm1_(double x) { return rc_expm1(x); }
    static double log_(double x) { return rc_log(x); }
    static double sqrt_(double x) { return sqrt(x); }
    static void sincos2pi_(double u, double *s, double *c) { rc_sincos2pi(u, s, c); }
    static double fma_(double a, double b, double c) { return fma(a, b, c); }
    static double lerp_(double a0, double a1, double w) { return rc_lerp(a0, a1, w); }
};

// ---------------------------------------------------------------- grid
struct Grid {
    int im, jm, km, sm;
    std::vector<float> x, xu, y, yu, z, zu;
};

// Gridn::mk_grid (definitions.h:68-136)
void mk_grid(const rc_params &p, int l, Grid &g) {
    const int im = p.maxi[l], jm = p.maxj[l], km = p.maxk[l], im0 = p.maxi[0];
    g.im = im;
    g.jm = jm;
    g.km = km;
    g.sm = p.maxs[l];
    g.x.assign(im + 2, 0.f);
    g.xu.assign(im + 1, 0.f);
    g.y.assign(jm + 2, 0.f);
    g.z.assign(km + 2, 0.f);
    g.yu.assign(jm + 1, 0.f);
    g.zu.assign(km + 1, 0.f);
    std::vector<float> xu0(im0 + 1);
    float dy = p.Ly * 1.0f / jm;
    float dz = p.Lz * 1.0f / km;
    for (int i = 0; i < jm + 1; i++) g.yu[i] = i * dy;
    for (int i = 0; i < km + 1; i++) g.zu[i] = i * dz;
    g.y[0] = -dy / 2;
    g.z[0] = -dz / 2;
    for (int i = 1; i < jm + 1; i++) g.y[i] = (g.yu[i - 1] + g.yu[i]) / 2;
    for (int i = 1; i < km + 1; i++) g.z[i] = (g.zu[i - 1] + g.zu[i]) / 2;
    g.y[jm + 1] = g.y[jm] + dy;
    g.z[km + 1] = g.z[km] + dz;
    xu0[0] = 0;
    for (int i = 1; i < im0 / 2 + 1; i++) {
        float r = (1.f * i) / im0;
        double rr = (double)r - 0.5;
        float dx = (float)(0.5 - p.fact_mesh * rr * rr);
        xu0[i] = xu0[i - 1] + dx;
    }
    float xnorm = xu0[im0 / 2];
    for (int i = 1; i < im0 / 2 + 1; i++) xu0[i] = (float)((double)p.Lx / 2. * xu0[i] / xnorm);
    for (int i = im0; i > im0 / 2; i--) xu0[i] = p.Lx - xu0[im0 - i];
    g.xu[0] = 0;
    for (int i = 1; i < im + 1; i++) g.xu[i] = xu0[(long long)i * im0 / im];
    for (int i = 1; i < im + 1; i++) g.x[i] = (float)(0.5 * (g.xu[i] + g.xu[i - 1]));
    g.x[0] = -g.x[1];
    g.x[im + 1] = g.xu[im] + (g.xu[im] - g.x[im]);
}

// tex3D(T, x, y, z) with linear filtering and clamp addressing
// (memory_copy_noint.cu:131-168), exact weights
float tex3(const std::vector<float> &T, int nx, int ny, int nz, float x, float y, float z) {
    float xb = x - 0.5f, yb = y - 0.5f, zb = z - 0.5f;
    float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    float ax = xb - fx, ay = yb - fy, az = zb - fz;
    int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    int i1 = std::min(std::max(i0 + 1, 0), nx - 1), j1 = std::min(std::max(j0 + 1, 0), ny - 1),
        k1 = std::min(std::max(k0 + 1, 0), nz - 1);
    i0 = std::min(std::max(i0, 0), nx - 1);
    j0 = std::min(std::max(j0, 0), ny - 1);
    k0 = std::min(std::max(k0, 0), nz - 1);
    auto at = [&](int i, int j, int k) { return T[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)]; };
    float c00 = at(i0, j0, k0) * (1.f - ax) + at(i1, j0, k0) * ax;
    float c10 = at(i0, j1, k0) * (1.f - ax) + at(i1, j1, k0) * ax;
    float c01 = at(i0, j0, k1) * (1.f - ax) + at(i1, j0, k1) * ax;
    float c11 = at(i0, j1, k1) * (1.f - ax) + at(i1, j1, k1) * ax;
    float c0 = c00 * (1.f - ay) + c10 * ay;
    float c1 = c01 * (1.f - ay) + c11 * ay;
    return c0 * (1.f - az) + c1 * az;
}

// Table coordinate with 8 fractional bits (the weight precision of the
// reference's texture filtering): q = rint(256 clamp((T - T0)/dT, 0, nT-1)).
template <typename R>
int tcoord(R T, R T0, R inv_dT, int nT) {
    R p = std::fmin(std::fmax((T - T0) * inv_dT, (R)0), (R)(nT - 1));
    return (int)std::rint(p * (R)256);
}

template <typename R>
R lerpq(const R *col, int nT, int q) {
    int i0 = q >> 8;
    int i1 = std::min(i0 + 1, nT - 1);
    R a = (R)(q & 255) * (R)0.00390625;
    return M<R>::lerp_(col[i0], col[i1], a);
}

template <typename R>
int find_idx(const R *cdf, int n, R u) {
    int lo = 0, w = n;
    while (w > lo + 1) {
        int d = (lo + w) / 2;
        if (u < cdf[d]) w = d;
        if (u >= cdf[d]) lo = d;
    }
    lo = lo + 1;
    if (u < cdf[0]) lo = 0;
    if (u == (R)1) lo = n - 1;
    return std::min(lo, n - 1);
}

// Wall band search edge rule.  0 (default): R below the wall CDF's own
// first entry selects band 0.  1: the reference's find_bandS test against
// the FLUID CDF's first entry probd[..][0] (mc_gpu_noint.cu:1189,1208), a
// defect this solver does not reproduce; the oracle offers it so the
// parity tests can measure what the defect does to the wall fluxes.
int g_ref_wall_edge = 0;

// Particle scattering tables of later solves (oracle_set_scattering), raw
// as the caller gave them: no scattering while nA == 0.  The march
// restates the device's scattering step (rc_device.cuh scatter_start,
// scatter_turn, march_step with SCAT): free path -ln(u) / k_s (none when
// k_s = 0), polar angle from the band's phase CDF (linear in angle between
// table angles), uniform azimuth, the standard rotation about the old
// direction; draws from the bundle's Philox counter with the event number in
// the fourth word.
struct ScatTables {
    int nB = 0, nQ = 0, nA = 0;
    std::vector<float> ksca, theta, cdf;
};
ScatTables g_scat;

template <typename R>
int find_idx_edge(const R *cdf, int n, R u, R edge0) {
    int lo = 0, w = n;
    while (w > lo + 1) {
        int d = (lo + w) / 2;
        if (u < cdf[d]) w = d;
        if (u >= cdf[d]) lo = d;
    }
    lo = lo + 1;
    if (u < edge0) lo = 0;
    if (u == (R)1) lo = n - 1;
    return std::min(lo, n - 1);
}

struct TraceSink {
    int max_cells = 0;
    int *cells = nullptr;
    int n = 0;
};

template <typename R>
struct Problem {
    rc_params p;
    int kloc = 0, nT = 0, nB = 0, nQ = 0;
    int wt[6];
    std::vector<Grid> grid;
    std::vector<std::vector<R>> gxu, gyu, gzu;  // faces as R
    std::vector<R> xc, yc, zc;
    std::vector<float> T;  // full field
    std::vector<std::vector<R>> Tl;                   // per level [km][jm][im]
    std::vector<std::vector<std::vector<R>>> Twl;     // per level, per wall
    std::vector<R> Tw0[2];                            // level-0 x-face temperatures [kmax][jmax]
    std::vector<R> kt, Ibt, probg, cdf_f, cdf_s, probq, Ibw, Tnb, kP, wvl, wvr, wvc, prob;
    int nA = 0;                      // scattering: table angles (0: no scattering)
    std::vector<R> ksca, pcdf, pth;  // [nB][nQ] scaled, [nB][nA] last = 1, [nA] turns
    oracle_setup su;
    R Tmax, Ibmax_f, Ibmax_w[2], T0, inv_dT;
    int row = 0;

    int init(const rc_params &pp, const rc_tables *t, const float *Tin) {
        p = pp;
        kloc = p.kmax / p.p_col;
        for (int w = 0; w < 6; ++w) {
            int b = p.bd[w];
            int ad = (w == RC_WEST) ? p.adiabw : (w == RC_EAST) ? p.adiabe : 0;
            wt[w] = (b == 2) ? (ad ? 6 : 2) : b;
        }
        const size_t nf = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
        T.assign(Tin, Tin + nf);
        grid.resize(p.grid_num);
        gxu.resize(p.grid_num);
        gyu.resize(p.grid_num);
        gzu.resize(p.grid_num);
        for (int l = 0; l < p.grid_num; ++l) {
            mk_grid(p, l, grid[l]);
            gxu[l].assign(grid[l].xu.begin(), grid[l].xu.end());
            gyu[l].assign(grid[l].yu.begin(), grid[l].yu.end());
            gzu[l].assign(grid[l].zu.begin(), grid[l].zu.end());
        }
        xc.assign(grid[0].x.begin(), grid[0].x.end());
        yc.assign(grid[0].y.begin(), grid[0].y.end());
        zc.assign(grid[0].z.begin(), grid[0].z.end());
        // Tmax: interior and x-wall face averages (mc_gpu_noint.cu:696-710)
        const int nx = p.imax + 2, ny = p.jmax + 2;
        auto at = [&](int i, int j, int k) { return T[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)]; };
        float tmax = 0.f, tmin = 3.4e38f;
        int status = 0;
        for (int k = 1; k < p.kmax + 1; k++)
            for (int j = 1; j < p.jmax + 1; j++) {
                for (int i = 1; i < p.imax + 1; i++) {
                    float v = at(i, j, k);
                    if (!std::isfinite(v)) {
                        status |= 2;
                        continue;
                    }
                    if (v <= 0.f) status |= 4;
                    tmax = std::max(tmax, v);
                    tmin = std::min(tmin, v);
                }
                float fw = (at(0, j, k) + at(1, j, k)) * 0.5f;
                float fe = (at(p.imax, j, k) + at(p.imax + 1, j, k)) * 0.5f;
                if (std::isfinite(fw)) tmax = std::max(tmax, fw);
                if (std::isfinite(fe)) tmax = std::max(tmax, fe);
            }
        Tmax = (R)tmax;
        // tables
        if (p.grey) {
            // read_tables.cpp:98-175
            nT = p.grey_nT;
            nB = p.grey_nB;
            nQ = 1;
            std::vector<float> l(nB), r(nB), c(nB);
            float dw = p.wvmax / nB;
            l[0] = 0;
            for (int i = 1; i < nB; i++) l[i] = l[i - 1] + dw;
            r[0] = dw;
            for (int i = 1; i < nB; i++) r[i] = r[i - 1] + dw;
            for (int i = 0; i < nB; i++) c[i] = (float)((double)(l[i] + r[i]) / 2.);
            wvl.assign(l.begin(), l.end());
            wvr.assign(r.begin(), r.end());
            wvc.assign(c.begin(), c.end());
            Tnb.resize(nT);
            for (int i = 0; i < nT; i++)
                Tnb[i] = (R)((double)p.Tmins * 0.9 + ((double)Tmax * 1.1 - (double)p.Tmins * 0.9) * (double)(R)i /
                             (double)(R)nT);
            kt.assign((size_t)nB * nT, (R)p.abscoeff);
            kP.assign(nT, (R)p.abscoeff);
            Ibt.resize((size_t)nB * nT);
            for (int b = 0; b < nB; ++b)
                for (int i = 0; i < nT; ++i) Ibt[(size_t)b * nT + i] = (R)rc_planck((double)Tnb[i], (double)wvc[b]);
            probg.assign((size_t)nT * nB, (R)1);
            probq.assign(1, (R)1);
        } else {
            if (!t) return RC_E_INVALID;
            nT = t->nT;
            nB = t->nB;
            nQ = t->nQ;
            // read_tables.cpp:21-96 (k and kP scaled by chanHeight)
            Tnb.resize(nT);
            kP.resize(nT);
            std::vector<float> ibf((size_t)nB * nT);
            for (int i = 0; i < nT; ++i) {
                Tnb[i] = (R)t->Tnb[i];
                kP[i] = (R)(float)((double)t->kP[i] * p.chanHeight);
            }
            kt.resize((size_t)nB * nQ * nT);
            for (int b = 0; b < nB; ++b)
                for (int g = 0; g < nQ; ++g)
                    for (int i = 0; i < nT; ++i)
                        kt[((size_t)b * nQ + g) * nT + i] =
                            (R)(float)((double)t->kq[((size_t)b * nT + i) * nQ + g] * p.chanHeight);
            Ibt.resize((size_t)nB * nT);
            for (int b = 0; b < nB; ++b)
                for (int i = 0; i < nT; ++i)
                    Ibt[(size_t)b * nT + i] = (R)(float)rc_planck((double)t->Tnb[i], (double)t->wvc[b]);
            probg.assign(t->probg, t->probg + (size_t)nT * nB * nQ);
            prob.assign(t->prob, t->prob + (size_t)nT * nB);
            wvl.assign(t->wvl, t->wvl + nB);
            wvr.assign(t->wvr, t->wvr + nB);
            wvc.assign(t->wvc, t->wvc + nB);
            // probq: cumulative g weights (mc_gpu_noint.cu:34-36)
            std::vector<float> pq(nQ);
            float cq = 0.f;
            for (int g = 0; g < nQ; ++g) {
                cq += t->wq[g];
                pq[g] = (g == nQ - 1) ? 1.0f : cq;
            }
            probq.assign(pq.begin(), pq.end());
        }
        Ibw.resize((size_t)6 * nB);
        for (int w = 0; w < 6; ++w)
            for (int b = 0; b < nB; ++b)
                Ibw[(size_t)w * nB + b] = (R)(float)rc_planck((double)p.Tw[w], (double)(float)wvc[b]);
        nA = 0;
        if (g_scat.nA > 0) {
            if (g_scat.nB != nB || g_scat.nQ != nQ) return RC_E_INVALID;
            nA = g_scat.nA;
            ksca.resize((size_t)nB * nQ);
            for (size_t i = 0; i < ksca.size(); ++i) ksca[i] = (R)rc_scatter_coef_scaled(g_scat.ksca[i], p.chanHeight);
            pcdf.resize((size_t)nB * nA);
            for (int b = 0; b < nB; ++b)
                for (int a = 0; a < nA; ++a)
                    pcdf[(size_t)b * nA + a] = (R)((a == nA - 1) ? 1.0f : g_scat.cdf[(size_t)b * nA + a]);
            pth.resize(nA);
            for (int a = 0; a < nA; ++a) pth[a] = (R)rc_angle_turns(g_scat.theta[a]);
        }
        // scalars: tm, row, kappamax, Ibmax (mc_gpu_noint.cu:74,820-826,1362-1366)
        int tm = (int)((Tmax - Tnb[0]) / (Tnb[1] - Tnb[0]));
        if (tm < 0) {
            tm = 0;
            status |= 1;
        }
        if (tm > nT - 2) {
            tm = nT - 2;
            status |= 1;
        }
        if ((R)tmin < Tnb[0] || Tmax > Tnb[nT - 1]) status |= 1;
        row = ((Tmax - Tnb[tm]) < (Tnb[tm + 1] - Tmax)) ? tm : tm + 1;
        R kappamax = p.grey ? (R)p.abscoeff
                            : (kP[tm + 1] - kP[tm]) / (Tnb[tm + 1] - Tnb[tm]) * (Tmax - Tnb[tm]) + kP[tm];
        R T4 = Tmax * Tmax * Tmax * Tmax;
        R kf = (R)4 * kappamax * T4;
        Ibmax_f = (R)((double)kf * p.stefan / (double)p.photmax);
        Ibmax_w[0] = (R)((double)p.eps[RC_WEST] * p.stefan * (double)T4 / (double)p.photmax);
        Ibmax_w[1] = (R)((double)p.eps[RC_EAST] * p.stefan * (double)T4 / (double)p.photmax);
        T0 = Tnb[0];
        inv_dT = (R)1 / (Tnb[1] - Tnb[0]);
        su.Tmax = tmax;
        su.Tmin = tmin;
        su.tm = tm;
        su.row = row;
        su.status = status;
        su.kappamax = (double)kappamax;
        su.Ibmax_f = (double)Ibmax_f;
        su.Ibmax_w[0] = (double)Ibmax_w[0];
        su.Ibmax_w[1] = (double)Ibmax_w[1];
        su.T0 = (double)T0;
        su.inv_dT = (double)inv_dT;
        // band CDF rows (find_band uses row tm or tm+1 of probd)
        cdf_f.resize(nB);
        cdf_s.resize(nB);
        auto planck_row = [&](std::vector<R> &o) {
            // read_tables.cpp:153-165 / :204-218
            R c = Ibt[(size_t)0 * nT + row] * (wvr[0] - wvl[0]) * (R)100;
            o[0] = c;
            for (int b = 1; b < nB; ++b) {
                c = c + Ibt[(size_t)b * nT + row] * (wvr[b] - wvl[b]) * (R)100;
                o[b] = c;
            }
            R last = o[nB - 1];
            for (int b = 0; b < nB; ++b) o[b] = o[b] / last;
        };
        if (p.grey) planck_row(cdf_f);
        else
            for (int b = 0; b < nB; ++b) cdf_f[b] = prob[(size_t)row * nB + b];
        if (p.calcwalls) planck_row(cdf_s);
        // temperature of every multigrid level at its cell centres
        // (mc_gpu_noint.cu:334-338), and wall emission temperatures
        const int nz = p.kmax + 2;
        Tl.resize(p.grid_num);
        Twl.assign(p.grid_num, std::vector<std::vector<R>>(6));
        for (int l = 0; l < p.grid_num; ++l) {
            const Grid &G = grid[l];
            const int rx = p.imax / G.im, ry = p.jmax / G.jm, rz = p.kmax / G.km;
            auto t1f = [&](int ic) { return ((float)ic - 0.5f) * (float)rx + 1.0f; };
            auto t2f = [&](int jc) { return ((float)jc - 0.5f) * (float)ry + 1.0f; };
            auto t3f = [&](int kc) { return ((float)kc - 0.5f) * (float)rz + 1.0f; };
            Tl[l].resize((size_t)G.im * G.jm * G.km);
            for (int kc = 1; kc <= G.km; ++kc)
                for (int jc = 1; jc <= G.jm; ++jc)
                    for (int ic = 1; ic <= G.im; ++ic)
                        Tl[l][((size_t)(kc - 1) * G.jm + (jc - 1)) * G.im + (ic - 1)] =
                            (R)tex3(T, nx, ny, nz, t1f(ic), t2f(jc), t3f(kc));
            for (int w = 0; w < 6; ++w) {
                if (wt[w] != 4 && wt[w] != 6) continue;
                const bool face = wt[w] == 6;
                std::vector<R> &A = Twl[l][w];
                if (w <= RC_EAST) {
                    float x = (w == RC_WEST) ? (face ? 1.0f : 1.5f) : (face ? (float)p.imax + 1.0f : (float)p.imax + 0.5f);
                    A.resize((size_t)G.jm * G.km);
                    for (int kc = 1; kc <= G.km; ++kc)
                        for (int jc = 1; jc <= G.jm; ++jc)
                            A[(size_t)(kc - 1) * G.jm + (jc - 1)] = (R)tex3(T, nx, ny, nz, x, t2f(jc), t3f(kc));
                } else if (w <= RC_NORTH) {
                    float y = (w == RC_SOUTH) ? (face ? 1.0f : 1.5f) : (face ? (float)p.jmax + 1.0f : (float)p.jmax + 0.5f);
                    A.resize((size_t)G.im * G.km);
                    for (int kc = 1; kc <= G.km; ++kc)
                        for (int ic = 1; ic <= G.im; ++ic)
                            A[(size_t)(kc - 1) * G.im + (ic - 1)] = (R)tex3(T, nx, ny, nz, t1f(ic), y, t3f(kc));
                } else {
                    float z = (w == RC_BOT) ? (face ? 1.0f : 1.5f) : (face ? (float)p.kmax + 1.0f : (float)p.kmax + 0.5f);
                    A.resize((size_t)G.im * G.jm);
                    for (int jc = 1; jc <= G.jm; ++jc)
                        for (int ic = 1; ic <= G.im; ++ic)
                            A[(size_t)(jc - 1) * G.im + (ic - 1)] = (R)tex3(T, nx, ny, nz, t1f(ic), t2f(jc), z);
                }
            }
        }
        for (int b = 0; b < 2; ++b) {
            Tw0[b].resize((size_t)p.jmax * p.kmax);
            float x = b == 0 ? 1.0f : (float)p.imax + 1.0f;
            for (int k = 1; k <= p.kmax; ++k)
                for (int j = 1; j <= p.jmax; ++j)
                    Tw0[b][(size_t)(k - 1) * p.jmax + (j - 1)] = (R)tex3(T, nx, ny, nz, x, (float)j + 0.5f, (float)k + 0.5f);
        }
        return RC_OK;
    }

    // ---- one bundle -------------------------------------------------
    struct Beam {
        int ic, jc, kc;
        R xp, yp, zp, sx, sy, sz, isx, isy, isz, tra;
        int flag[3];
        // scattering: counter words of the bundle, events so far, the
        // scattering coefficient of its band and g point, distance left to
        // the next event
        uint32_t cx, cy, cz;
        int nev;
        R ks, dist;
    };

    // Absorption along ds (mc_gpu_noint.cu:358-370).
    void absorb(Beam &ray, double &De, R ds, R absco, R blackpow, R Ibmax, R ratioI, R invTi4, R tol) const {
        R em = M<R>::expm1_(-(ds * absco));
        R alpha = -em;
        R dI = M<R>::fma_(invTi4, blackpow, (R)-1);
        R c = Ibmax * ray.tra;
        c = c * alpha;
        c = c * ratioI;
        c = c * dI;
        De -= (double)c;
        ray.tra = M<R>::fma_(ray.tra, em, ray.tra);
        if (ray.tra < tol) {
            R c2 = (Ibmax * ray.tra) * ratioI;
            c2 = c2 * dI;
            De -= (double)c2;
            ray.tra = 0;
        }
    }

    // New direction at the next scattering event of a bundle in band nb and
    // the optical depth to the event after it.
    void scatter_turn(Beam &ray, int nb) const {
        ray.nev += 1;
        rc_u32x4 c = {ray.cx, ray.cy, ray.cz, (uint32_t)(ray.nev + 1)};
        rc_u32x4 d = rc_philox4x32_10(c, (uint32_t)p.seed, (uint32_t)(p.seed >> 32));
        R u_t = (R)rc_u01(d.x), u_p = (R)rc_u01(d.y), u_s = (R)rc_u01(d.z);
        const R *cdf = &pcdf[(size_t)nb * nA];
        int lo = 0, hi = nA - 1;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (u_t < cdf[mid]) hi = mid;
            else lo = mid;
        }
        R c0 = cdf[hi - 1], c1 = cdf[hi];
        R fr = (c1 > c0) ? (u_t - c0) / (c1 - c0) : (R)0;
        if (fr > (R)1) fr = (R)1;
        R t0 = pth[hi - 1], t1 = pth[hi];
        R th = M<R>::fma_(fr, t1 - t0, t0);
        R st, ct, sp, cp;
        M<R>::sincos2pi_(th, &st, &ct);
        M<R>::sincos2pi_(u_p, &sp, &cp);
        R nx, ny, nz;
        if (std::fabs(ray.sz) > (R)0.99999) {
            nx = st * cp;
            ny = st * sp;
            nz = (ray.sz > (R)0) ? ct : -ct;
        } else {
            R w = M<R>::sqrt_((R)1 - ray.sz * ray.sz);
            R a = st / w;
            nx = a * (ray.sx * ray.sz * cp - ray.sy * sp) + ray.sx * ct;
            ny = a * (ray.sy * ray.sz * cp + ray.sx * sp) + ray.sy * ct;
            nz = ray.sz * ct - st * cp * w;
        }
        if (nx == (R)0) nx = (R)1e-10;
        if (ny == (R)0) ny = (R)1e-10;
        if (nz == (R)0) nz = (R)1e-10;
        ray.sx = nx;
        ray.sy = ny;
        ray.sz = nz;
        ray.isx = (R)1 / nx;
        ray.isy = (R)1 / ny;
        ray.isz = (R)1 / nz;
        ray.flag[0] = ray.sx < 0;
        ray.flag[1] = ray.sy < 0;
        ray.flag[2] = ray.sz < 0;
        ray.dist = -M<R>::log_(u_s) / ray.ks;
    }

    R Tcell(int lev, int ic, int jc, int kc) const {
        const Grid &G = grid[lev];
        return Tl[lev][((size_t)(kc - 1) * G.jm + (jc - 1)) * G.im + (ic - 1)];
    }

    void deposit(Beam &ray, double &De, R Ibmax, R ratioI, R invTi4, R e) const {
        R c = (Ibmax * ray.tra) * M<R>::fma_(invTi4, e, (R)-1);
        c = c * ratioI;
        De -= (double)c;
        ray.tra = 0;
    }

    void wall(Beam &ray, double &De, int lev, int w, int nb, const R *ibcol, R Ibmax, R ratioI, R invTi4) const {
        const Grid &G = grid[lev];
        switch (wt[w]) {
            case 1:  // periodic
                if (w == RC_WEST) { ray.ic = G.im; ray.xp = (R)p.Lx; }
                else if (w == RC_EAST) { ray.ic = 1; ray.xp = 0; }
                else if (w == RC_SOUTH) { ray.jc = G.jm; ray.yp = (R)p.Ly; }
                else if (w == RC_NORTH) { ray.jc = 1; ray.yp = 0; }
                else if (w == RC_BOT) { ray.kc = G.km; ray.zp = (R)p.Lz; }
                else { ray.kc = 1; ray.zp = 0; }
                break;
            case 2:
                deposit(ray, De, Ibmax, ratioI, invTi4, Ibw[(size_t)w * nB + nb]);
                break;
            case 4:
            case 6: {
                int idx;
                if (w <= RC_EAST) idx = (ray.kc - 1) * G.jm + (ray.jc - 1);
                else if (w <= RC_NORTH) idx = (ray.kc - 1) * G.im + (ray.ic - 1);
                else idx = (ray.jc - 1) * G.im + (ray.ic - 1);
                R Tw = Twl[lev][w][idx];
                deposit(ray, De, Ibmax, ratioI, invTi4, lerpq(ibcol, nT, tcoord(Tw, T0, inv_dT, nT)));
                break;
            }
            case 3: {  // specular reflection, on the component normal to the wall
                if (w == RC_WEST || w == RC_EAST) {
                    ray.xp = (w == RC_WEST) ? (R)0 : (R)p.Lx;
                    ray.sx = -ray.sx;
                    ray.isx = -ray.isx;
                    ray.ic = (w == RC_WEST) ? 1 : G.im;
                    ray.flag[0] = ray.sx < 0;
                } else if (w == RC_SOUTH || w == RC_NORTH) {
                    ray.yp = (w == RC_SOUTH) ? (R)0 : (R)p.Ly;
                    ray.sy = -ray.sy;
                    ray.isy = -ray.isy;
                    ray.jc = (w == RC_SOUTH) ? 1 : G.jm;
                    ray.flag[1] = ray.sy < 0;
                } else {
                    ray.zp = (w == RC_BOT) ? (R)0 : (R)p.Lz;
                    ray.sz = -ray.sz;
                    ray.isz = -ray.isz;
                    ray.kc = (w == RC_BOT) ? 1 : G.km;
                    ray.flag[2] = ray.sz < 0;
                }
                break;
            }
            default:
                ray.tra = 0;
        }
    }

    // march_ray (mc_gpu_noint.cu:245-658) on level lev until tra <= tol or
    // the step budget of the level is spent
    int march(Beam &ray, double &De, int lev, int nb, const R *kcol, const R *ibcol, R Ibmax, R ratioI, R invTi4,
              R tol, TraceSink *ts) const {
        const Grid &G = grid[lev];
        const std::vector<R> &xu = gxu[lev], &yu = gyu[lev], &zu = gzu[lev];
        int counter = 0;
        while ((ray.tra > tol) && (counter < G.sm)) {
            if (ts && ts->n < ts->max_cells) {
                int *c = ts->cells + (size_t)ts->n * 4;
                c[0] = lev;
                c[1] = ray.ic;
                c[2] = ray.jc;
                c[3] = ray.kc;
            }
            if (ts) ts->n++;
            R fxu = xu[ray.ic - ray.flag[0]], fyu = yu[ray.jc - ray.flag[1]], fzu = zu[ray.kc - ray.flag[2]];
            R dsx = (fxu - ray.xp) * ray.isx;
            R dsy = (fyu - ray.yp) * ray.isy;
            R dsz = (fzu - ray.zp) * ray.isz;
            R tf = Tcell(lev, ray.ic, ray.jc, ray.kc);
            int q = tcoord(tf, T0, inv_dT, nT);
            R absco = lerpq(kcol, nT, q);
            R blackpow = lerpq(ibcol, nT, q);
            R ds = dsx;
            if (ds > dsy) ds = dsy;
            if (ds > dsz) ds = dsz;
            if (nA > 0) {
                if (ds > ray.dist) {
                    // the next scattering event lies inside this cell
                    R dsc = ray.dist;
                    ray.xp = M<R>::fma_(dsc, ray.sx, ray.xp);
                    ray.yp = M<R>::fma_(dsc, ray.sy, ray.yp);
                    ray.zp = M<R>::fma_(dsc, ray.sz, ray.zp);
                    absorb(ray, De, dsc, absco, blackpow, Ibmax, ratioI, invTi4, tol);
                    scatter_turn(ray, nb);
                    counter += 1;
                    continue;
                }
                ray.dist = ray.dist - ds;
            }
            if (ds == dsx) ray.xp = fxu;
            else ray.xp = M<R>::fma_(ds, ray.sx, ray.xp);
            if (ds == dsy) ray.yp = fyu;
            else ray.yp = M<R>::fma_(ds, ray.sy, ray.yp);
            if (ds == dsz) ray.zp = fzu;
            else ray.zp = M<R>::fma_(ds, ray.sz, ray.zp);
            absorb(ray, De, ds, absco, blackpow, Ibmax, ratioI, invTi4, tol);
            int axis;
            if (dsx < dsy) axis = (dsx < dsz) ? 0 : 2;
            else axis = (dsy < dsz) ? 1 : 2;
            if (axis == 0) {
                if (ray.flag[0]) {
                    ray.ic = ray.ic - 1;
                    if (ray.ic == 0) wall(ray, De, lev, RC_WEST, nb, ibcol, Ibmax, ratioI, invTi4);
                } else {
                    ray.ic = ray.ic + 1;
                    if (ray.ic == G.im + 1) wall(ray, De, lev, RC_EAST, nb, ibcol, Ibmax, ratioI, invTi4);
                }
            } else if (axis == 1) {
                if (ray.flag[1]) {
                    ray.jc = ray.jc - 1;
                    if (ray.jc == 0) wall(ray, De, lev, RC_SOUTH, nb, ibcol, Ibmax, ratioI, invTi4);
                } else {
                    ray.jc = ray.jc + 1;
                    if (ray.jc == G.jm + 1) wall(ray, De, lev, RC_NORTH, nb, ibcol, Ibmax, ratioI, invTi4);
                }
            } else {
                if (ray.flag[2]) {
                    ray.kc = ray.kc - 1;
                    if (ray.kc == 0) wall(ray, De, lev, RC_BOT, nb, ibcol, Ibmax, ratioI, invTi4);
                } else {
                    ray.kc = ray.kc + 1;
                    if (ray.kc == G.km + 1) wall(ray, De, lev, RC_TOP, nb, ibcol, Ibmax, ratioI, invTi4);
                }
            }
            counter += 1;
        }
        return counter;
    }

    // One bundle of cell (i,j,k) [kind 0] or wall cell (j,k) [kind 1,2].
    double bundle(int kind, int i, int j, int k, int v, int h, rc_trace_rec *rec, TraceSink *ts,
                  long long *steps) const {
        uint32_t cell = (kind == 0) ? (uint32_t)((i - 1) + p.imax * ((j - 1) + p.jmax * (k - 1)))
                                    : (uint32_t)((j - 1) + p.jmax * (k - 1));
        rc_u32x4 ctr = {(uint32_t)h, (uint32_t)v | ((uint32_t)kind << 24), cell, 0u};
        rc_u32x4 d = rc_philox4x32_10(ctr, (uint32_t)p.seed, (uint32_t)(p.seed >> 32));
        R u_phi = (R)rc_u01(d.x), u_mu = (R)rc_u01(d.y), u_b = (R)rc_u01(d.z), u_g = (R)rc_u01(d.w);
        R sp, cp;
        M<R>::sincos2pi_(u_phi, &sp, &cp);
        Beam ray;
        ray.tra = 1;
        int nb, g;
        R Ti, Ibmax, tol;
        if (kind == 0) {
            R mu = (R)1 - (R)2 * u_mu;
            R st = M<R>::sqrt_(((R)1 - mu) * ((R)1 + mu));
            ray.sx = mu;
            ray.sy = st * cp;
            ray.sz = st * sp;
            if (ray.sx == 0) ray.sx = (R)1e-10;
            if (ray.sy == 0) ray.sy = (R)1e-10;
            if (ray.sz == 0) ray.sz = (R)1e-10;
            ray.xp = xc[i];
            ray.yp = yc[j];
            ray.zp = zc[k];
            ray.ic = i;
            ray.jc = j;
            ray.kc = k;
            nb = find_idx(cdf_f.data(), nB, u_b);
            g = (nQ > 1) ? find_idx(&probg[((size_t)row * nB + nb) * nQ], nQ, u_g) : 0;
            Ti = Tcell(0, i, j, k);
            Ibmax = Ibmax_f;
            tol = (R)p.toll;
        } else {
            int bound = kind - 1;
            R st;
            if (bound == 0) {
                ray.sx = M<R>::sqrt_((R)1 - u_mu);
                st = M<R>::sqrt_(u_mu);
            } else {
                ray.sx = -M<R>::sqrt_(u_mu);
                st = M<R>::sqrt_((R)1 - u_mu);
            }
            ray.sy = st * cp;
            ray.sz = st * sp;
            if (std::fabs(ray.sx) <= (R)1e-10) ray.sx = (R)(1 - 2 * bound) * (R)1e-10;
            if (std::fabs(ray.sy) <= (R)1e-10) ray.sy = (R)((ray.sy > 0) - (ray.sy <= 0)) * (R)1e-10;
            if (std::fabs(ray.sz) <= (R)1e-10) ray.sz = (R)((ray.sz > 0) - (ray.sz <= 0)) * (R)1e-10;
            ray.xp = bound == 0 ? (R)0 : (R)p.Lx;
            ray.yp = yc[j];
            ray.zp = zc[k];
            ray.ic = bound == 0 ? 1 : p.imax;
            ray.jc = j;
            ray.kc = k;
            nb = g_ref_wall_edge ? find_idx_edge(cdf_s.data(), nB, u_b, cdf_f[0]) : find_idx(cdf_s.data(), nB, u_b);
            g = (nQ > 1) ? find_idx(probq.data(), nQ, u_g) : 0;
            Ti = Tw0[bound][(size_t)(k - 1) * p.jmax + (j - 1)];
            Ibmax = Ibmax_w[bound];
            tol = (R)p.tollS;
        }
        ray.flag[0] = ray.sx < 0;
        ray.flag[1] = ray.sy < 0;
        ray.flag[2] = ray.sz < 0;
        ray.isx = (R)1 / ray.sx;
        ray.isy = (R)1 / ray.sy;
        ray.isz = (R)1 / ray.sz;
        // scattering: the bundle's counter words, its coefficient and the
        // optical depth to its first event (draw 1)
        ray.cx = ctr.x;
        ray.cy = ctr.y;
        ray.cz = ctr.z;
        ray.nev = 0;
        ray.ks = (nA > 0) ? ksca[(size_t)nb * nQ + g] : (R)0;
        ray.dist = (R)3.0e38f;
        if (ray.ks > (R)0) {
            rc_u32x4 c1 = {ctr.x, ctr.y, ctr.z, 1u};
            rc_u32x4 d1 = rc_philox4x32_10(c1, (uint32_t)p.seed, (uint32_t)(p.seed >> 32));
            ray.dist = -M<R>::log_((R)rc_u01(d1.x)) / ray.ks;
        }
        if (rec) {
            rec->nb = nb;
            rec->g = g;
            rec->sx = (float)ray.sx;
            rec->sy = (float)ray.sy;
            rec->sz = (float)ray.sz;
            rec->nsteps = 0;
            rec->end_level = 0;
            rec->tra = 0.f;
            rec->De = 0.0;
        }
        const R *kcol = &kt[((size_t)nb * nQ + g) * nT];
        const R *ibcol = &Ibt[(size_t)nb * nT];
        // OERM weights: ratioI = Ib(Ti) k(Ti) / (Ib(Tmax) k(Tmax)) for the fluid
        // (mc_gpu_noint.cu:180-186), Ib(Ti)/Ib(Tmax) for walls (:1421-1424)
        int pos_i = tcoord(Ti, T0, inv_dT, nT), pos_m = tcoord(Tmax, T0, inv_dT, nT);
        R Ib_i = lerpq(ibcol, nT, pos_i);
        if (!(Ib_i > 0)) return 0.0;
        R invTi4 = (R)1 / Ib_i;
        R ratioI;
        if (kind == 0) {
            R k_i = lerpq(kcol, nT, pos_i);
            R den = lerpq(ibcol, nT, pos_m) * lerpq(kcol, nT, pos_m);
            if (!(den > 0)) return 0.0;
            ratioI = (Ib_i * k_i) / den;
        } else {
            R Ib_m = lerpq(ibcol, nT, pos_m);
            if (!(Ib_m > 0)) return 0.0;
            ratioI = Ib_i / Ib_m;
            const Grid &G = grid[0];
            if (ray.flag[0] && ray.xp == (R)G.xu[ray.ic - 1]) ray.ic = ray.ic - 1;
            if (ray.flag[1] && ray.yp == (R)G.yu[ray.jc - 1]) ray.jc = ray.jc - 1;
            if (ray.flag[2] && ray.zp == (R)G.zu[ray.kc - 1]) ray.kc = ray.kc - 1;
            if (!ray.flag[0] && ray.xp == (R)G.xu[ray.ic]) ray.ic = ray.ic + 1;
            if (!ray.flag[1] && ray.yp == (R)G.yu[ray.jc]) ray.jc = ray.jc + 1;
            if (!ray.flag[2] && ray.zp == (R)G.zu[ray.kc]) ray.kc = ray.kc + 1;
        }
        double De = 0.0;
        int nsteps = 0, last_lev = 0;
        for (int grd = 0; grd < p.grid_num; grd++) {
            int n = march(ray, De, grd, nb, kcol, ibcol, Ibmax, ratioI, invTi4, tol, ts);
            if (n > 0) last_lev = grd;
            nsteps += n;
            if (grd < p.grid_num - 1) {
                // coarsen the cell index (mc_gpu_noint.cu:215-223)
                int rx = grid[grd].im / grid[grd + 1].im, ry = grid[grd].jm / grid[grd + 1].jm,
                    rz = grid[grd].km / grid[grd + 1].km;
                ray.ic = (ray.ic + rx - 1) / rx;
                ray.jc = (ray.jc + ry - 1) / ry;
                ray.kc = (ray.kc + rz - 1) / rz;
            }
            if (!(ray.tra > tol)) break;
        }
        if (steps) *steps += nsteps;
        if (rec) {
            rec->nsteps = nsteps;
            rec->end_level = last_lev;
            rec->tra = (float)ray.tra;
            rec->De = De;
        }
        return De;
    }

    // work decomposition of the device (chunks of rpt bundles)
    void decompose(int rpt, int &nchunk, int &gsize, int &nparts) const {
        int nc = (p.photmax + rpt - 1) / rpt;
        if (nc <= 32) {
            int p2 = 1;
            while (p2 < nc) p2 <<= 1;
            nc = p2;
            gsize = nc;
            nparts = 1;
        } else {
            nc = (nc + 31) / 32 * 32;
            gsize = 32;
            nparts = nc / 32;
        }
        nchunk = nc;
    }

    // replicate sum of one (cell, v) in the device's summation order
    double replicate(int kind, int i, int j, int k, int v, int rpt, long long *steps) const {
        int nchunk, gsize, nparts;
        decompose(rpt, nchunk, gsize, nparts);
        double Dv = 0.0;
        for (int part = 0; part < nparts; ++part) {
            double P = 0.0;
            for (int q = part * gsize; q < (part + 1) * gsize; ++q) {
                double s = 0.0;
                for (int ho = 0; ho < rpt; ++ho) {
                    int h = q * rpt + ho;
                    double De = (h < p.photmax) ? bundle(kind, i, j, k, v, h, nullptr, nullptr, steps) : 0.0;
                    s += De;
                }
                P += s;
            }
            Dv += P;
        }
        return Dv;
    }

    // mean and variance of the mean over nVar replicates (:234-239)
    void cell_stats(int kind, int i, int j, int k, int rpt, double &mean, double &var, long long *steps) const {
        const int nVar = p.nVar;
        std::vector<double> Dv(nVar);
        double sum = 0.0;
        for (int v = 0; v < nVar; ++v) {
            Dv[v] = replicate(kind, i, j, k, v, rpt, steps);
            sum += Dv[v];
        }
        mean = sum / nVar;
        var = 0.0;
        if (nVar > 1) {
            double a = 1. / (nVar - 0.5);
            a = a * 1. / (nVar - 1);
            for (int v = 0; v < nVar; ++v) {
                double d = Dv[v] - mean;
                var += a * d * d;
            }
        }
    }
};

template <typename R>
int solve_t(const rc_params *p, const rc_tables *t, const float *T, int zstart, int rpt, long long cb, long long ce,
            int do_walls, int nthreads, double *q64, double *var64, double *qw64, double *vw64, double *steps,
            double *bundles) {
    Problem<R> P;
    int rc = P.init(*p, t, T);
    if (rc) return rc;
    const int kloc = P.kloc;
    const long long ncf = (long long)p->imax * p->jmax * kloc;
    if (ce < 0 || ce > ncf) ce = ncf;
    if (cb < 0) cb = 0;
    long long tot_steps = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : tot_steps)
#endif
    for (long long c = cb; c < ce; ++c) {
        int i = (int)(c % p->imax) + 1;
        long long r = c / p->imax;
        int j = (int)(r % p->jmax) + 1;
        int k = (int)(r / p->jmax) + zstart;
        double m, v;
        long long st = 0;
        P.cell_stats(0, i, j, k, rpt, m, v, &st);
        tot_steps += st;
        if (q64) q64[c] = m;
        if (var64) var64[c] = v;
    }
    long long nb = (ce - cb) * (long long)p->nVar * p->photmax;
    if (do_walls && p->calcwalls) {
        const long long nwc = (long long)p->jmax * kloc;
        for (int b = 0; b < 2; ++b) {
            if ((b == 0 && !p->adiabw) || (b == 1 && !p->adiabe)) continue;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : tot_steps)
#endif
            for (long long c = 0; c < nwc; ++c) {
                int j = (int)(c % p->jmax) + 1;
                int k = (int)(c / p->jmax) + zstart;
                double m, v;
                long long st = 0;
                P.cell_stats(1 + b, 0, j, k, rpt, m, v, &st);
                tot_steps += st;
                if (qw64) qw64[b * nwc + c] = m;
                if (vw64) vw64[b * nwc + c] = v;
            }
            nb += nwc * (long long)p->nVar * p->photmax;
        }
    }
    if (steps) *steps = (double)tot_steps;
    if (bundles) *bundles = (double)nb;
    return RC_OK;
}

template <typename R>
int trace_t(const rc_params *p, const rc_tables *t, const float *T, int n, const rc_bundle_id *ids,
                   rc_trace_rec *out, int max_cells, int *cells) {
    Problem<R> P;
    int rc = P.init(*p, t, T);
    if (rc) return rc;
    for (int b = 0; b < n; ++b) {
        TraceSink ts;
        ts.max_cells = cells ? max_cells : 0;
        ts.cells = cells ? cells + (size_t)b * max_cells * 4 : nullptr;
        if (ts.cells)
            for (int q = 0; q < max_cells * 4; ++q) ts.cells[q] = -1;
        const rc_bundle_id &id = ids[b];
        P.bundle(id.kind, id.i, id.j, id.k, id.v, id.h, &out[b], &ts, nullptr);
    }
    return RC_OK;
}


}  // namespace

extern "C" {

int oracle_solve(const rc_params *p, const rc_tables *t, const float *T, int zstart, int rpt, long long cell_begin,
                 long long cell_end, int do_walls, int fp64, int nthreads, double *q64, double *var64, double *qw64,
                 double *vw64, double *steps, double *bundles) {
    if (!p || !T || rpt < 1) return RC_E_INVALID;
    if (fp64)
        return solve_t<double>(p, t, T, zstart, rpt, cell_begin, cell_end, do_walls, nthreads, q64, var64, qw64, vw64,
                               steps, bundles);
    return solve_t<float>(p, t, T, zstart, rpt, cell_begin, cell_end, do_walls, nthreads, q64, var64, qw64, vw64,
                          steps, bundles);
}

int oracle_trace(const rc_params *p, const rc_tables *t, const float *T, int zstart, int fp64, int n,
                 const rc_bundle_id *ids, rc_trace_rec *out, int max_cells, int *cells) {
    (void)zstart;
    if (!p || !T || (n > 0 && (!ids || !out))) return RC_E_INVALID;
    if (fp64) return trace_t<double>(p, t, T, n, ids, out, max_cells, cells);
    return trace_t<float>(p, t, T, n, ids, out, max_cells, cells);
}

int oracle_setup_scalars(const rc_params *p, const rc_tables *t, const float *T, int fp64, oracle_setup *out) {
    if (!p || !T || !out) return RC_E_INVALID;
    if (fp64) {
        Problem<double> P;
        int rc = P.init(*p, t, T);
        *out = P.su;
        return rc;
    }
    Problem<float> P;
    int rc = P.init(*p, t, T);
    *out = P.su;
    return rc;
}

// Band and g point of emission for given uniforms (find_band / find_bandS,
// mc_gpu_noint.cu:1103-1233, with the edge rule chosen by
// oracle_set_ref_wall_edge for walls), and the CDF rows they search:
// cdf_f / cdf_s [nB] (fluid / wall band CDF at the table row nearest
// Tmax), probq [nQ]; any output may be NULL.
int oracle_sample_bands(const rc_params *p, const rc_tables *t, const float *T, int kind, int n, const float *u_b,
                        const float *u_g, int *nb, int *g, float *cdf_f, float *cdf_s, float *probq, int *row) {
    if (!p || !T || kind < 0 || kind > 2) return RC_E_INVALID;
    Problem<float> P;
    int rc = P.init(*p, t, T);
    if (rc) return rc;
    const int nB = P.nB, nQ = P.nQ;
    for (int i = 0; i < n; ++i) {
        int b, q;
        if (kind == 0) {
            b = find_idx(P.cdf_f.data(), nB, u_b[i]);
            q = nQ > 1 ? find_idx(&P.probg[((size_t)P.su.row * nB + b) * nQ], nQ, u_g[i]) : 0;
        } else {
            b = g_ref_wall_edge ? find_idx_edge(P.cdf_s.data(), nB, u_b[i], P.cdf_f[0])
                                : find_idx(P.cdf_s.data(), nB, u_b[i]);
            q = nQ > 1 ? find_idx(P.probq.data(), nQ, u_g[i]) : 0;
        }
        nb[i] = b;
        g[i] = q;
    }
    if (cdf_f) memcpy(cdf_f, P.cdf_f.data(), nB * sizeof(float));
    if (cdf_s && !P.cdf_s.empty()) memcpy(cdf_s, P.cdf_s.data(), nB * sizeof(float));
    if (probq) memcpy(probq, P.probq.data(), nQ * sizeof(float));
    if (row) *row = P.su.row;
    return RC_OK;
}

int oracle_grid_level(const rc_params *p, int level, float *xu, float *yu, float *zu, float *x, float *y, float *z) {
    if (!p || level < 0 || level >= p->grid_num) return RC_E_INVALID;
    Grid g;
    mk_grid(*p, level, g);
    auto cp = [](float *d, const std::vector<float> &s) {
        if (d) memcpy(d, s.data(), s.size() * sizeof(float));
    };
    cp(xu, g.xu);
    cp(yu, g.yu);
    cp(zu, g.zu);
    cp(x, g.x);
    cp(y, g.y);
    cp(z, g.z);
    return RC_OK;
}

int oracle_level_T(const rc_params *p, const float *T, int level, float *out) {
    if (!p || !T || !out || level < 0 || level >= p->grid_num) return RC_E_INVALID;
    const int nx = p->imax + 2, ny = p->jmax + 2, nz = p->kmax + 2;
    std::vector<float> TT(T, T + (size_t)nx * ny * nz);
    const int im = p->maxi[level], jm = p->maxj[level], km = p->maxk[level];
    const int rx = p->imax / im, ry = p->jmax / jm, rz = p->kmax / km;
    for (int kc = 1; kc <= km; ++kc)
        for (int jc = 1; jc <= jm; ++jc)
            for (int ic = 1; ic <= im; ++ic)
                out[((size_t)(kc - 1) * jm + (jc - 1)) * im + (ic - 1)] =
                    tex3(TT, nx, ny, nz, ((float)ic - 0.5f) * (float)rx + 1.0f, ((float)jc - 0.5f) * (float)ry + 1.0f,
                         ((float)kc - 0.5f) * (float)rz + 1.0f);
    return RC_OK;
}

}  // extern "C"

// Exposes the shared arithmetic primitives to the tests (Philox and the
// exp/expm1/sincos/Planck/log functions of radchan_math.h).
extern "C" int oracle_math_probe(int which, int n, const double *in, double *out) {
    for (int i = 0; i < n; ++i) {
        const double x = in[i];
        switch (which) {
            case 0: out[i] = (double)rc_expf((float)x); break;
            case 1: out[i] = (double)rc_expm1f((float)x); break;
            case 2: out[i] = rc_exp(x); break;
            case 3: out[i] = rc_expm1(x); break;
            case 4: { float s, c; rc_sincos2pif((float)x, &s, &c); out[2 * i] = s; out[2 * i + 1] = c; break; }
            case 5: { double s, c; rc_sincos2pi(x, &s, &c); out[2 * i] = s; out[2 * i + 1] = c; break; }
            case 6: out[i] = rc_planck(x, in[n + i]); break;
            case 7: out[i] = (double)rc_logf((float)x); break;
            case 8: out[i] = rc_log(x); break;
            default: return RC_E_INVALID;
        }
    }
    return RC_OK;
}

extern "C" int oracle_philox(const unsigned int *ctr, const unsigned int *key, unsigned int *out) {
    rc_u32x4 c = {ctr[0], ctr[1], ctr[2], ctr[3]};
    rc_u32x4 r = rc_philox4x32_10(c, key[0], key[1]);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
    return RC_OK;
}

// ---------------------------------------------------------------------------
// Seeded synthetic correlated-k tables, restated from the table recipe of the
// benchmark configurations so that the oracle's inputs need nothing from the
// product library:
//   k_{b,g}(T) = k0_b exp(kexp xi_g) (T/1000)^{n_b},
//   log10 k0_b ~ U[logk_lo, logk_hi], n_b ~ U[-nexp, nexp] (Philox draws),
//   xi_g / w_g the nQ-point Gauss-Legendre rule on [-1, 1] (w_g/2 as g
//   weights), band centres ~ U[nu_lo, nu_hi] sorted with edges at midpoints,
//   nT uniformly spaced temperatures on [T_lo, T_hi];
//   band CDF ~ sum_g w_g k I_b dnu and g CDF ~ w_g k (nbcorrk/calc_prob.cpp
//   :404-453), Planck mean pi sum k I_b dnu / (sigma T^4), and k_avg of the
//   last temperature row (read_tables.cpp:52 overwrites it per row).
// Outputs: caller arrays in the rc_tables layout (kq [nB][nT][nQ], prob
// [nT][nB], probg [nT][nB][nQ]).
// ---------------------------------------------------------------------------
namespace {
double draw_u53(uint64_t seed, uint32_t stream, uint32_t idx) {
    rc_u32x4 c = {idx, stream, 0x5eedu, 0u};
    const rc_u32x4 r = rc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t hi = r.x >> 5, lo = r.y >> 6;  // 27 + 26 bits
    return (double)(hi * 67108864ull + lo) * (1.0 / 9007199254740992.0);
}

// Gauss-Legendre nodes (ascending) and weights by Newton's method on P_n.
void gl_rule(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = cos(RC_PI_D * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            dp = n * (z * p1 - p2) / (z * z - 1.0);
            const double z0 = z;
            z = z0 - p1 / dp;
            if (fabs(z - z0) < 1e-15) break;
        }
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}
}  // namespace

// Scattering tables for the oracle's later solves and traces (NULL: none).
// The same checks as the library's rc_scattering_validate are left to the
// callers (tests); dimensions must match the solve's bands and g points.
extern "C" int oracle_set_scattering(const rc_scattering *s) {
    g_scat = ScatTables();
    if (!s) return 0;
    if (s->nB < 1 || s->nQ < 1 || s->nA < 2 || !s->ksca || !s->theta || !s->phase_cdf) return RC_E_INVALID;
    g_scat.nB = s->nB;
    g_scat.nQ = s->nQ;
    g_scat.nA = s->nA;
    g_scat.ksca.assign(s->ksca, s->ksca + (size_t)s->nB * s->nQ);
    g_scat.theta.assign(s->theta, s->theta + s->nA);
    g_scat.cdf.assign(s->phase_cdf, s->phase_cdf + (size_t)s->nB * s->nA);
    return 0;
}

extern "C" int oracle_set_ref_wall_edge(int on) {
    g_ref_wall_edge = on ? 1 : 0;
    return 0;
}

extern "C" int oracle_tables_synthetic(const rc_synth_spec *s, float *Tnb, float *kP, float *wvl, float *wvr,
                                       float *wvc, float *kavg, float *kq, float *prob, float *probg, float *wq) {
    if (!s || s->nB < 1 || s->nQ < 1 || s->nT < 2 || !(s->T_hi > s->T_lo) || !(s->T_lo > 0) ||
        !(s->nu_hi > s->nu_lo) || !(s->nu_lo > 0))
        return -1;
    const int nB = s->nB, nQ = s->nQ, nT = s->nT;
    std::vector<double> xi, wgl;
    gl_rule(nQ, xi, wgl);
    std::vector<double> wg(nQ);
    for (int g = 0; g < nQ; ++g) {
        wg[g] = wgl[g] / 2.0;
        wq[g] = (float)wg[g];
    }
    std::vector<double> nu(nB), k0(nB), ne(nB), el(nB), er(nB);
    for (int b = 0; b < nB; ++b) nu[b] = s->nu_lo + (s->nu_hi - s->nu_lo) * draw_u53(s->seed, 1, b);
    std::sort(nu.begin(), nu.end());
    for (int b = 0; b < nB; ++b) {
        k0[b] = pow(10.0, s->logk_lo + (s->logk_hi - s->logk_lo) * draw_u53(s->seed, 2, b));
        ne[b] = -s->nexp + 2.0 * s->nexp * draw_u53(s->seed, 3, b);
    }
    for (int b = 0; b < nB; ++b) {
        el[b] = b == 0 ? s->nu_lo : 0.5 * (nu[b - 1] + nu[b]);
        er[b] = b == nB - 1 ? s->nu_hi : 0.5 * (nu[b] + nu[b + 1]);
        wvl[b] = (float)el[b];
        wvr[b] = (float)er[b];
        wvc[b] = (float)nu[b];
    }
    const double sigma = 5.670373e-08;
    std::vector<double> kg(nQ), pband(nB);
    for (int i = 0; i < nT; ++i) {
        const double T = s->T_lo + (s->T_hi - s->T_lo) * i / (double)(nT - 1);
        Tnb[i] = (float)T;
        double total = 0.0;
        for (int b = 0; b < nB; ++b) {
            const double ib = rc_planck(T, nu[b]);
            const double dnu = (er[b] - el[b]) * 100.0;
            double kav = 0.0, pb = 0.0, sg = 0.0;
            for (int g = 0; g < nQ; ++g) {
                kg[g] = k0[b] * exp(s->kexp * xi[g]) * pow(T / 1000.0, ne[b]);
                kq[((size_t)b * nT + i) * nQ + g] = (float)kg[g];
                kav += wg[g] * kg[g];
                pb += wg[g] * kg[g] * ib * dnu;
            }
            if (i == nT - 1) kavg[b] = (float)kav;
            pband[b] = pb;
            total += pb;
            for (int g = 0; g < nQ; ++g) sg += kg[g] * wg[g];
            double cg = 0.0;
            for (int g = 0; g < nQ; ++g) {
                cg += kg[g] * wg[g];
                probg[((size_t)i * nB + b) * nQ + g] = g == nQ - 1 ? 1.0f : (float)(cg / sg);
            }
        }
        kP[i] = (float)(RC_PI_D * total / (sigma * T * T * T * T));
        double c = 0.0;
        for (int b = 0; b < nB; ++b) {
            c += pband[b];
            prob[(size_t)i * nB + b] = b == nB - 1 ? 1.0f : (float)(c / total);
        }
    }
    return 0;
}
