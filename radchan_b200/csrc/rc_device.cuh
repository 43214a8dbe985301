// rc_device.cuh -- sm_100a device code of the OERM Monte Carlo solver.
//
// Reference: src/montecarlo/mc_gpu_noint.cu
//   kernel_fluid   :55-243   per-cell bundle emission + OERM tally
//   march_ray      :245-658  multigrid ray march with the wall conditions
//   find_band(S)   :1103-1233 band / g-point bisection
//   emiss_ang(S)   :1077-1102 emission directions
//   kernel_surface :1316-1482 wall-flux kernel
//   kernel_results :1296-1314 copy-out
//
// Arithmetic contract (shared with the CPU oracle, which restates the same
// operations in the same order so that sampled bands, g points, visited
// cells and per-bundle tallies agree bit for bit):
//   * no FMA contraction (nvcc -fmad=false); explicit fmaf() only inside
//     radchan_math.h;
//   * face distance ds = (face - p) * (1/s), the reciprocal formed once per
//     direction change;
//   * table coordinate p = clamp((T - T0) * (1/dT), 0, nT-1), stored per cell
//     of every multigrid level; v = col[i0]*(1-a) + col[i1]*a with i0 = (int)p,
//     a = p - i0;
//   * alpha = -expm1(-(ds*k)), tra *= (1 + expm1(-(ds*k)));
//   * step tally c = (((Ibmax*tra)*alpha)*ratioI)*(invTi4*Ib - 1) in the
//     march precision, accumulated into an FP64 bundle sum;
//   * per-bundle sums are added in bundle order within a chunk of
//     rays_per_thread bundles, chunk sums in chunk order, and replicate
//     sums in replicate order, whatever thread traced which bundle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "radchan.h"
#include "radchan_math.h"

namespace rc {

constexpr int kWarp = 32;
constexpr int kRing = 64;  // per-warp ring of emitted bundles (two waves)

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
template <typename R>
struct DLevel {
    int im, jm, km, maxs;
    int rx, ry, rz, pad;      // ratio to the next (coarser) level
    const R *xu, *yu, *zu;    // faces
    const R *P;               // [km][jm][im] table coordinate of the cell temperature
    const R *Pw[6];           // wall emission temperature coordinates (or null)
};

// Per-solve scalars written on the device by the set-up kernels.
struct DScalars {
    unsigned int tmax_bits;   // float bits of max T (non-negative)
    unsigned int tmin_bits;   // float bits of min T
    int status;               // bit 0 out of table, bit 1 non-finite, bit 2 T <= 0
    int tm, row;
    int pad;
    double Tmax, kappamax, Ibmax_f, Ibmax_w[2];
    double T0, inv_dT;        // first table temperature and 1/spacing
    double Pm;                // table coordinate of Tmax
    unsigned long long steps, bundles;
};

template <typename R>
struct DSolve {
    DLevel<R> lev[RC_MAX_LEVELS];
    int nlev;
    int imax, jmax, kmax, kloc, kfirst;
    int wtype[6];
    int nT, nB, nQ;
    int nVar, photmax, rpt, nchunk, gsize, nparts;
    int nwalls, wall_id[2];
    int pad;
    R Lx, Ly, Lz;
    R toll, tollS;
    // run-time values (copied from DScalars by the kernels)
    R Pm, Ibmax_f, Ibmax_w0, Ibmax_w1;
    int row, pad2;
    const R *xc, *yc, *zc;    // level-0 cell centres incl. ghosts
    const R *kt;              // [nB][nQ][nT]
    const R *Ibt;             // [nB][nT]
    const R *probg;           // [nT][nB][nQ]
    const R *cdf_f;           // [nB] fluid band CDF at the selected row
    const R *cdf_s;           // [nB] wall band CDF at the selected row
    const R *probq;           // [nQ]
    const R *Ibw;             // [6][nB] fixed wall spectra
    const R *Pw0[2];          // level-0 west/east face coordinates [kmax][jmax]
    DScalars *sc;
    double *partial;
    long long n_fluid_items, n_items, n_tiles;
    uint32_t key0, key1;
};

// ---------------------------------------------------------------------------
// precision traits
// ---------------------------------------------------------------------------
template <typename R> struct RT;
template <> struct RT<float> {
    static __device__ __forceinline__ float expm1_(float x) { return rc_expm1f(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ void sincos2pi_(float u, float *s, float *c) { rc_sincos2pif(u, s, c); }
    static __device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fabs_(float a) { return fabsf(a); }
};
template <> struct RT<double> {
    static __device__ __forceinline__ double expm1_(double x) { return rc_expm1(x); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ void sincos2pi_(double u, double *s, double *c) { rc_sincos2pi(u, s, c); }
    static __device__ __forceinline__ double fmin_(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double fmax_(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double fabs_(double a) { return fabs(a); }
};

// Table coordinate of a temperature: clamp((T - T0)/dT, 0, nT-1); NaN -> 0.
template <typename R>
__device__ __forceinline__ R table_coord(R T, R T0, R inv_dT, int nT) {
    return RT<R>::fmin_(RT<R>::fmax_((T - T0) * inv_dT, (R)0), (R)(nT - 1));
}

// Linear interpolation in temperature along one table column at a clamped
// coordinate (the reference does this with a clamped linear-filter texture,
// mc_gpu_noint.cu:341-345, memory_copy_noint.cu:241-245).
struct Lerp {
    int i0, i1;
};
template <typename R>
__device__ __forceinline__ R lerp_at(const R *col, int i0, int i1, R a) {
    return col[i0] * ((R)1 - a) + col[i1] * a;
}
template <typename R>
__device__ __forceinline__ R tab_lerp(const R *col, int nT, R p) {
    const int i0 = (int)p;
    const int i1 = min(i0 + 1, nT - 1);
    return lerp_at(col, i0, i1, p - (R)i0);
}

// Inverse-CDF bisection with the reference's edge rules
// (mc_gpu_noint.cu:1113-1127): R < cdf[0] -> 0, R == 1 -> n-1.
template <typename R>
__device__ __forceinline__ int bisect(const R *cdf, int n, R u) {
    int lo = 0, w = n;
    while (w > lo + 1) {
        int d = (lo + w) >> 1;
        if (u < cdf[d]) w = d;
        else lo = d;
    }
    int r = lo + 1;
    if (u < cdf[0]) r = 0;
    if (u == (R)1) r = n - 1;
    return min(r, n - 1);
}

// A bundle after emission: direction, sampled band/g and OERM weights.
template <typename R>
struct Emitted {
    R sx, sy, sz, isx, isy, isz, ratioI, invTi4;
    int nbg;   // nb | g << 20
    int b;     // index in the warp's bundle pool
};

template <typename R>
struct Ray {
    R xp, yp, zp;
    R sx, sy, sz;
    R isx, isy, isz;
    R tra;
    R Ibmax, ratioI, invTi4, tol;
    const R *kcol, *ibcol;
    int ic, jc, kc;
    int fx, fy, fz;
    int lev, counter;
    int nb;
    double De;
};

// Philox counter of one bundle: (h, v | kind << 24, cell, 0).
__device__ __forceinline__ rc_u32x4 bundle_draws(uint32_t key0, uint32_t key1, int h, int v, int kind, uint32_t cell) {
    rc_u32x4 c;
    c.x = (uint32_t)h;
    c.y = (uint32_t)v | ((uint32_t)kind << 24);
    c.z = cell;
    c.w = 0u;
    return rc_philox4x32_10(c, key0, key1);
}

// Emission of one bundle.  kind 0: fluid cell (i,j,k) (kernel_fluid
// :115-186); kind 1/2: west/east wall cell (j,k) (kernel_surface
// :1381-1424).  Returns false if the bundle carries no energy.
template <typename R>
__device__ __forceinline__ bool emit_bundle(Emitted<R> &e, const DSolve<R> &S, int kind, int i, int j, int k, int v,
                                            int h) {
    const uint32_t cell = (kind == 0)
                              ? (uint32_t)((i - 1) + S.imax * ((j - 1) + S.jmax * (k - 1)))
                              : (uint32_t)((j - 1) + S.jmax * (k - 1));
    rc_u32x4 d = bundle_draws(S.key0, S.key1, h, v, kind, cell);
    const R u_phi = (R)rc_u01(d.x), u_mu = (R)rc_u01(d.y), u_b = (R)rc_u01(d.z), u_g = (R)rc_u01(d.w);
    R sp, cp;
    RT<R>::sincos2pi_(u_phi, &sp, &cp);
    R Pi;
    int nb, g;
    if (kind == 0) {
        // isotropic: cos(theta) = 1 - 2u (emiss_ang, :1077-1084)
        const R mu = (R)1 - (R)2 * u_mu;
        const R st = RT<R>::sqrt_(((R)1 - mu) * ((R)1 + mu));
        e.sx = mu;
        e.sy = st * cp;
        e.sz = st * sp;
        if (e.sx == (R)0) e.sx = (R)1e-10;  // :132-137
        if (e.sy == (R)0) e.sy = (R)1e-10;
        if (e.sz == (R)0) e.sz = (R)1e-10;
        nb = bisect(S.cdf_f, S.nB, u_b);
        g = (S.nQ > 1) ? bisect(S.probg + ((size_t)S.row * S.nB + nb) * S.nQ, S.nQ, u_g) : 0;
        const DLevel<R> &L0 = S.lev[0];
        Pi = L0.P[((k - 1) * L0.jm + (j - 1)) * L0.im + (i - 1)];
    } else {
        // Lambertian: theta = acos(1 - 2u)/2 (+pi/2 on the east wall)
        // (emiss_angS, :1093-1102), i.e. cos = sqrt(1-u) / -sqrt(u).
        const int bound = kind - 1;
        R st;
        if (bound == 0) {
            e.sx = RT<R>::sqrt_((R)1 - u_mu);
            st = RT<R>::sqrt_(u_mu);
        } else {
            e.sx = -RT<R>::sqrt_(u_mu);
            st = RT<R>::sqrt_((R)1 - u_mu);
        }
        e.sy = st * cp;
        e.sz = st * sp;
        if (RT<R>::fabs_(e.sx) <= (R)1e-10) e.sx = (R)(1 - 2 * bound) * (R)1e-10;  // :1395-1400
        if (RT<R>::fabs_(e.sy) <= (R)1e-10) e.sy = (R)((e.sy > (R)0) - (e.sy <= (R)0)) * (R)1e-10;
        if (RT<R>::fabs_(e.sz) <= (R)1e-10) e.sz = (R)((e.sz > (R)0) - (e.sz <= (R)0)) * (R)1e-10;
        nb = bisect(S.cdf_s, S.nB, u_b);
        g = (S.nQ > 1) ? bisect(S.probq, S.nQ, u_g) : 0;
        Pi = S.Pw0[bound][(k - 1) * S.jmax + (j - 1)];
    }
    e.nbg = nb | (g << 20);
    e.isx = (R)1 / e.sx;
    e.isy = (R)1 / e.sy;
    e.isz = (R)1 / e.sz;
    // OERM weights (:180-186 fluid, :1421-1424 walls)
    const R *kcol = S.kt + ((size_t)nb * S.nQ + g) * S.nT;
    const R *ibcol = S.Ibt + (size_t)nb * S.nT;
    const R Ib_i = tab_lerp(ibcol, S.nT, Pi);
    const R Ib_m = tab_lerp(ibcol, S.nT, S.Pm);
    if (!(Ib_i > (R)0) || !(Ib_m > (R)0)) return false;
    e.invTi4 = (R)1 / Ib_i;
    if (kind == 0) {
        const R k_i = tab_lerp(kcol, S.nT, Pi);
        const R k_m = tab_lerp(kcol, S.nT, S.Pm);
        if (!(k_m > (R)0)) return false;
        e.ratioI = ((((R)1 / e.invTi4) / Ib_m) * k_i) / k_m;
    } else {
        e.ratioI = ((R)1 / e.invTi4) / Ib_m;
    }
    return true;
}

// Position, cell and weights of an emitted bundle at its start point.
template <typename R>
__device__ __forceinline__ void place_bundle(Ray<R> &r, const DSolve<R> &S, const Emitted<R> &e, int kind, int i,
                                             int j, int k) {
    r.sx = e.sx;
    r.sy = e.sy;
    r.sz = e.sz;
    r.isx = e.isx;
    r.isy = e.isy;
    r.isz = e.isz;
    r.ratioI = e.ratioI;
    r.invTi4 = e.invTi4;
    const int nb = e.nbg & 0xfffff, g = e.nbg >> 20;
    r.nb = nb;
    r.kcol = S.kt + ((size_t)nb * S.nQ + g) * S.nT;
    r.ibcol = S.Ibt + (size_t)nb * S.nT;
    r.fx = r.sx < (R)0;
    r.fy = r.sy < (R)0;
    r.fz = r.sz < (R)0;
    r.lev = 0;
    r.counter = 0;
    r.tra = (R)1;
    r.De = 0.0;
    r.jc = j;
    r.kc = k;
    r.yp = S.yc[j];
    r.zp = S.zc[k];
    if (kind == 0) {
        r.ic = i;
        r.xp = S.xc[i];
        r.Ibmax = S.Ibmax_f;
        r.tol = S.toll;
    } else {
        const int bound = kind - 1;
        r.ic = (bound == 0) ? 1 : S.imax;
        r.xp = (bound == 0) ? (R)0 : S.Lx;
        r.Ibmax = bound == 0 ? S.Ibmax_w0 : S.Ibmax_w1;
        r.tol = S.tollS;
        // cell shift when the start point lies on a face (:1429-1441)
        const DLevel<R> &G = S.lev[0];
        if (r.fx && r.xp == G.xu[r.ic - 1]) r.ic = r.ic - 1;
        if (r.fy && r.yp == G.yu[r.jc - 1]) r.jc = r.jc - 1;
        if (r.fz && r.zp == G.zu[r.kc - 1]) r.kc = r.kc - 1;
        if (!r.fx && r.xp == G.xu[r.ic]) r.ic = r.ic + 1;
        if (!r.fy && r.yp == G.yu[r.jc]) r.jc = r.jc + 1;
        if (!r.fz && r.zp == G.zu[r.kc]) r.kc = r.kc + 1;
    }
}

// Deposit the remaining energy on a black wall emitting Ib_wall
// (:398-399 and its siblings): De -= Ibmax*tra*(invTi4*e - 1)*ratioI.
template <typename R>
__device__ __forceinline__ void wall_deposit(Ray<R> &r, R e) {
    R c = (r.Ibmax * r.tra) * (r.invTi4 * e - (R)1);
    c = c * r.ratioI;
    r.De -= (double)c;
    r.tra = (R)0;
}

// Wall condition for wall w at level L (:375-654, with the y/z specular
// branches reflecting the right component and flag).
template <typename R>
__device__ __forceinline__ void hit_wall(Ray<R> &r, const DSolve<R> &S, const DLevel<R> &L, int w) {
    const int t = S.wtype[w];
    if (t == 1) {  // periodic
        switch (w) {
            case RC_WEST: r.ic = L.im; r.xp = S.Lx; break;
            case RC_EAST: r.ic = 1; r.xp = (R)0; break;
            case RC_SOUTH: r.jc = L.jm; r.yp = S.Ly; break;
            case RC_NORTH: r.jc = 1; r.yp = (R)0; break;
            case RC_BOT: r.kc = L.km; r.zp = S.Lz; break;
            default: r.kc = 1; r.zp = (R)0; break;
        }
    } else if (t == 2) {  // black wall at its own temperature
        wall_deposit(r, S.Ibw[(size_t)w * S.nB + r.nb]);
    } else if (t == 4 || t == 6) {  // black wall at a field temperature
        int idx;
        if (w <= RC_EAST) idx = (r.kc - 1) * L.jm + (r.jc - 1);
        else if (w <= RC_NORTH) idx = (r.kc - 1) * L.im + (r.ic - 1);
        else idx = (r.jc - 1) * L.im + (r.ic - 1);
        wall_deposit(r, tab_lerp(r.ibcol, S.nT, L.Pw[w][idx]));
    } else if (t == 3) {  // specular
        switch (w) {
            case RC_WEST: r.xp = (R)0; r.sx = -r.sx; r.isx = -r.isx; r.ic = 1; r.fx = r.sx < (R)0; break;
            case RC_EAST: r.xp = S.Lx; r.sx = -r.sx; r.isx = -r.isx; r.ic = L.im; r.fx = r.sx < (R)0; break;
            case RC_SOUTH: r.yp = (R)0; r.sy = -r.sy; r.isy = -r.isy; r.jc = 1; r.fy = r.sy < (R)0; break;
            case RC_NORTH: r.yp = S.Ly; r.sy = -r.sy; r.isy = -r.isy; r.jc = L.jm; r.fy = r.sy < (R)0; break;
            case RC_BOT: r.zp = (R)0; r.sz = -r.sz; r.isz = -r.isz; r.kc = 1; r.fz = r.sz < (R)0; break;
            default: r.zp = S.Lz; r.sz = -r.sz; r.isz = -r.isz; r.kc = L.km; r.fz = r.sz < (R)0; break;
        }
    } else {  // lost ray
        r.tra = (R)0;
    }
}

// One ray-cell crossing (one iteration of the while loop of march_ray,
// :252-656).
template <typename R>
__device__ __forceinline__ void march_step(Ray<R> &r, const DSolve<R> &S, const DLevel<R> &L) {
    const R fxu = L.xu[r.ic - r.fx];
    const R fyu = L.yu[r.jc - r.fy];
    const R fzu = L.zu[r.kc - r.fz];
    const R p = __ldg(&L.P[((r.kc - 1) * L.jm + (r.jc - 1)) * L.im + (r.ic - 1)]);
    const R dsx = (fxu - r.xp) * r.isx;
    const R dsy = (fyu - r.yp) * r.isy;
    const R dsz = (fzu - r.zp) * r.isz;
    const int i0 = (int)p;
    const int i1 = min(i0 + 1, S.nT - 1);
    const R a = p - (R)i0;
    const R absco = lerp_at(r.kcol, i0, i1, a);
    const R blackpow = lerp_at(r.ibcol, i0, i1, a);
    R ds = dsx;
    if (ds > dsy) ds = dsy;
    if (ds > dsz) ds = dsz;
    r.xp = (ds == dsx) ? fxu : r.xp + ds * r.sx;
    r.yp = (ds == dsy) ? fyu : r.yp + ds * r.sy;
    r.zp = (ds == dsz) ? fzu : r.zp + ds * r.sz;
    const R em = RT<R>::expm1_(-(ds * absco));
    const R alpha = -em;
    const R dI = r.invTi4 * blackpow - (R)1;
    R c = r.Ibmax * r.tra;
    c = c * alpha;
    c = c * r.ratioI;
    c = c * dI;
    r.De -= (double)c;
    r.tra = r.tra * ((R)1 + em);
    if (r.tra < r.tol) {  // cutoff: deposit the rest here (:365-370)
        R c2 = (r.Ibmax * r.tra) * r.ratioI;
        c2 = c2 * dI;
        r.De -= (double)c2;
        r.tra = (R)0;
    }
    int axis;
    if (dsx < dsy) axis = (dsx < dsz) ? 0 : 2;
    else axis = (dsy < dsz) ? 1 : 2;
    int w = -1;
    if (axis == 0) {
        if (r.fx) { if (--r.ic == 0) w = RC_WEST; }
        else { if (++r.ic == L.im + 1) w = RC_EAST; }
    } else if (axis == 1) {
        if (r.fy) { if (--r.jc == 0) w = RC_SOUTH; }
        else { if (++r.jc == L.jm + 1) w = RC_NORTH; }
    } else {
        if (r.fz) { if (--r.kc == 0) w = RC_BOT; }
        else { if (++r.kc == L.km + 1) w = RC_TOP; }
    }
    if (w >= 0) hit_wall(r, S, L, w);
    r.counter += 1;
}

// Advance to coarser levels while the step budget of the current level is
// spent (:210-224).  Returns false when the ray must stop (budget of the
// last level spent).
template <typename R>
__device__ __forceinline__ bool level_advance(Ray<R> &r, const DSolve<R> &S) {
    while (r.counter >= S.lev[r.lev].maxs) {
        if (r.lev >= S.nlev - 1) return false;
        const DLevel<R> &L = S.lev[r.lev];
        r.ic = (r.ic + L.rx - 1) / L.rx;
        r.jc = (r.jc + L.ry - 1) / L.ry;
        r.kc = (r.kc + L.rz - 1) / L.rz;
        r.lev += 1;
        r.counter = 0;
    }
    return true;
}

// Decoded work item: item = ((cell*nVar + v)*nchunk + q); the wall items
// follow the fluid items.  kind = -1 marks an item past the end.
struct ItemId {
    int kind, i, j, k, v, h0;
};

template <typename R>
__device__ __forceinline__ ItemId decode_item(const DSolve<R> &S, long long item) {
    ItemId d;
    d.kind = -1;
    d.i = d.j = d.k = d.v = d.h0 = 0;
    if (item >= S.n_items) return d;
    long long it = item;
    int kind = 0;
    if (it >= S.n_fluid_items) {
        it -= S.n_fluid_items;
        kind = 1;
    }
    const int q = (int)(it % S.nchunk);
    const long long t = it / S.nchunk;
    d.v = (int)(t % S.nVar);
    const long long c = t / S.nVar;
    d.h0 = q * S.rpt;
    if (kind == 0) {
        d.i = (int)(c % S.imax) + 1;
        const long long cj = c / S.imax;
        d.j = (int)(cj % S.jmax) + 1;
        d.k = (int)(cj / S.jmax) + S.kfirst;
        d.kind = 0;
    } else {
        const long long nwc = (long long)S.jmax * S.kloc;
        const int slot = (int)(c / nwc);
        const long long wc = c % nwc;
        d.j = (int)(wc % S.jmax) + 1;
        d.k = (int)(wc / S.jmax) + S.kfirst;
        d.kind = 1 + S.wall_id[slot];
    }
    return d;
}

}  // namespace rc
