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
//   * no automatic FMA contraction (nvcc -fmad=false, g++ -ffp-contract=off);
//     every fused multiply-add is written out (fma_ here, the same call in
//     the oracle, fmaf() in radchan_math.h), so both sides round alike;
//   * face distance ds = (face - p) * (1/s), the reciprocal formed once per
//     direction change; positions p = fma(ds, s, p) on the axes not crossed;
//   * table coordinate q = rint(256 * clamp((T - T0) * (1/dT), 0, nT-1)),
//     8 fractional bits (the weight precision of the texture unit the
//     reference interpolates with), stored as uint16 per cell of every
//     multigrid level; v = fma(col[i1], a, col[i0]*(1-a)) (rc_lerpf) with
//     i0 = q >> 8, i1 = min(i0 + 1, nT - 1), a = (q & 255) / 256;
//   * em = expm1(-(ds*k)), alpha = -em, tra = fma(tra, em, tra);
//   * step tally c = (((Ibmax*tra)*alpha)*ratioI)*fma(invTi4, Ib, -1) in the
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
constexpr int kRing = 64;    // per-warp ring of emitted bundles (two waves)
constexpr int kGuide = 256;  // buckets of the band-CDF guide tables
constexpr int kFeedIdle = 14; // idle lanes that make a warp leave its step loop to take new bundles
constexpr int kTurnGather = 5; // lanes waiting at scattering events that make a warp draw their turns
constexpr int kChunkMax = 8;  // tiles a warp claims per work-queue fetch (guided: fewer near the end)
constexpr int kPhaseGuide = 64;  // phase-CDF guide buckets per band (scattering turns)

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
template <typename R>
struct DLevel {
    int im, jm, km, maxs;
    int rx, ry, rz;           // ratio to the next (coarser) level
    unsigned mrx, mry, mrz;   // floor(2^32 / r) + 1 (0 for r = 1): (n + r - 1) / r as a multiply-high
    const R *xu, *yu, *zu;    // faces (views into DSolve::faces)
    const uint16_t *P;        // table coordinate of every cell, i fastest (see cell_index);
                              // a view into DSolve::Pall
    const uint16_t *Pw[6];    // wall emission temperature coordinates (or null)
};

// Interleaved table row: k and I_b at temperature rows t and t+1 (the last
// row repeats itself), so one 16-byte load serves a step's interpolation.
template <typename R>
struct alignas(4 * sizeof(R)) KIRow {
    R k0, ib0, k1, ib1;
};

// Per-solve scalars written on the device by the set-up kernels.
struct DScalars {
    unsigned int tmax_bits;   // float bits of max T (non-negative)
    unsigned int tmin_bits;   // float bits of min T
    int status;               // bit 0 out of table, bit 1 non-finite, bit 2 T <= 0, bit 3 index out of bounds
    int tm, row;
    int bad_site;             // first out-of-bounds site (bounds-checked build)
    double Tmax, kappamax, Ibmax_f, Ibmax_w[2];
    double T0, inv_dT;        // first table temperature and 1/spacing
    int Pm;                   // table coordinate of Tmax
    int pad2;
    unsigned long long steps, bundles;
};

template <typename R>
struct DSolve {
    // what a step reads of its level, two 16-byte loads:
    // lva = offsets of xu, yu, zu in faces and of the coordinates in Pall;
    // lvb = (im, jm, km, maxs)
    int4 lva[RC_MAX_LEVELS], lvb[RC_MAX_LEVELS];
    const R *faces;           // every level's xu | yu | zu, one after the other
    const uint16_t *Pall;     // every level's table coordinates, one after the other
    DLevel<R> lev[RC_MAX_LEVELS];
    int nlev;
    int imax, jmax, kmax, kloc, kfirst;
    int wtype[6];
    int nT, nB, nQ;
    int nVar, photmax, rpt, nchunk, gsize, nparts;
    int sort;  // 1: emitted bundles enter the ring in ascending k (band-sorted order)
    int nwalls, wall_id[2];
    int pad;
    R Lx, Ly, Lz;
    R toll, tollS;
    // run-time values (copied from DScalars by the kernels)
    R Ibmax_f, Ibmax_w0, Ibmax_w1;
    int Pm, row;
    const R *xc, *yc, *zc;    // level-0 cell centres incl. ghosts
    const R *kt;              // [nB][nQ][nT]
    const R *Ibt;             // [nB][nT]
    const R *probg;           // [nT][nB][nQ]
    const R *cdf_f;           // [nB] fluid band CDF at the selected row
    const R *cdf_s;           // [nB] wall band CDF at the selected row
    const R *probq;           // [nQ]
    const R *Ibw;             // [6][nB] fixed wall spectra
    const uint16_t *Pw0[2];   // level-0 west/east face coordinates [kmax][jmax]
    const KIRow<R> *ki;       // [nB][nQ][nT] interleaved k / I_b rows
    const R *den_f;           // [nB][nQ] I_b(Tmax) k(Tmax) (fluid OERM weight denominator)
    const R *ibm;             // [nB] I_b(Tmax) (wall OERM weight denominator)
    const int *guide_f;       // [kGuide] first band with cdf_f > q/kGuide
    const int *guide_s;       // [kGuide] same for cdf_s
    // scattering particles (nA = 0: none)
    const R *ksca;            // [nB][nQ] scattering coefficient (scaled by chanHeight)
    const R *pcdf;            // [nB][nA] cumulative phase-function probability, last = 1
    const R *pth;             // [nA] scattering angles in turns (theta / 2 pi)
    const uint16_t *pguide;   // [nB][kPhaseGuide+1] phase-CDF search brackets (phase_index)
    int nA;
    int pad3;
    DScalars *sc;
    double *partial;
    long long n_fluid_items, n_items, n_tiles;
    // multiply-high reciprocals of the item decomposition divisors
    unsigned long long mg_nchunk, mg_nvar, mg_imax, mg_jmax, mg_nwc;
    unsigned long long nwc;   // jmax * kloc
    uint32_t key0, key1;
    long long tile_base;      // first tile of this launch within the solve (server quanta)
    // extents for the bounds-checked build
    long long n_faces, n_P, n_partial;
};

// Bounds-checked indexing.  The product build compiles RC_IX to the plain
// index.  A build with RC_CHECKED=1 (libradchan_checked.so) checks every
// table, field and partial-sum index of the march against its array's
// extent: an index outside [0, n) sets status bit 3 and the first offending
// site in DScalars::bad_site, and is replaced by 0 so the access stays
// inside the array.  Nothing traps.
#ifndef RC_CHECKED
#define RC_CHECKED 0
#endif
enum RcSite : int {
    SITE_FACE = 1, SITE_PYRAMID, SITE_ROW, SITE_IBW, SITE_WALL_T, SITE_WALL_ROW, SITE_CENTRE, SITE_EMIT_T,
    SITE_WALL_EMIT_T, SITE_FACE_SHIFT, SITE_EMIT_ROW, SITE_DEN, SITE_IBM, SITE_PROBG, SITE_PARTIAL, SITE_LEVEL,
    SITE_CDF, SITE_KSCA, SITE_PHASE
};
#if RC_CHECKED
__device__ __forceinline__ long long rc_ix(long long i, long long n, int site, DScalars *sc) {
    if (i >= 0 && i < n) return i;
    atomicOr(&sc->status, 8);
    atomicCAS(&sc->bad_site, 0, site);
    return 0;
}
#define RC_IX(i, n, site, S) rc_ix((long long)(i), (long long)(n), (site), (S).sc)
#else
#define RC_IX(i, n, site, S) (i)
#endif

// ---------------------------------------------------------------------------
// precision traits
// ---------------------------------------------------------------------------
template <typename R> struct RT;
template <> struct RT<float> {
    static __device__ __forceinline__ float expm1_(float x) { return rc_expm1f(x); }
    static __device__ __forceinline__ float log_(float x) { return rc_logf(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float lerp_(float a0, float a1, float w) { return rc_lerpf(a0, a1, w); }
    static __device__ __forceinline__ void sincos2pi_(float u, float *s, float *c) { rc_sincos2pif(u, s, c); }
    static __device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fabs_(float a) { return fabsf(a); }
};
template <> struct RT<double> {
    static __device__ __forceinline__ double expm1_(double x) { return rc_expm1(x); }
    static __device__ __forceinline__ double log_(double x) { return rc_log(x); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
    static __device__ __forceinline__ double lerp_(double a0, double a1, double w) { return rc_lerp(a0, a1, w); }
    static __device__ __forceinline__ void sincos2pi_(double u, double *s, double *c) { rc_sincos2pi(u, s, c); }
    static __device__ __forceinline__ double fmin_(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double fmax_(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double fabs_(double a) { return fabs(a); }
};

// Table coordinate of a temperature with 8 fractional bits, the weight
// precision of the texture unit the reference interpolates with:
// q = rint(256 * clamp((T - T0)/dT, 0, nT-1)); NaN -> 0.  nT <= 256.
template <typename R>
__device__ __forceinline__ int table_coord(R T, R T0, R inv_dT, int nT) {
    const R p = RT<R>::fmin_(RT<R>::fmax_((T - T0) * inv_dT, (R)0), (R)(nT - 1));
    return (int)rint(p * (R)256);
}

// One interleaved table row through the read-only path.
__device__ __forceinline__ KIRow<float> load_row(const KIRow<float> *p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    KIRow<float> r;
    r.k0 = v.x;
    r.ib0 = v.y;
    r.k1 = v.z;
    r.ib1 = v.w;
    return r;
}
__device__ __forceinline__ KIRow<double> load_row(const KIRow<double> *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    KIRow<double> r;
    r.k0 = a.x;
    r.ib0 = a.y;
    r.k1 = b.x;
    r.ib1 = b.y;
    return r;
}

// Fraction of a table coordinate: (q mod 256) / 256, exact.
template <typename R>
__device__ __forceinline__ R coord_frac(int q) {
    return (R)(q & 255) * (R)0.00390625;
}

// Offset of cell (i,j,k) (1-based) in an im x jm x km array, i fastest.
// (A 4x4x4-brick layout was measured 2-3% slower: its index arithmetic
// costs more issue slots than its locality saves in L1 misses.)
__device__ __forceinline__ int cell_index(int i, int j, int k, int im, int jm) {
    return (i - 1) + im * ((j - 1) + jm * (k - 1));
}

// Linear interpolation in temperature along one table column at a clamped
// coordinate (the reference does this with a clamped linear-filter texture,
// mc_gpu_noint.cu:341-345, memory_copy_noint.cu:241-245).
template <typename R>
__device__ __forceinline__ R lerp_at(const R *col, int i0, int i1, R a) {
    return RT<R>::lerp_(col[i0], col[i1], a);
}
template <typename R>
__device__ __forceinline__ R tab_lerp(const R *col, int nT, int q) {
    const int i0 = q >> 8;
    const int i1 = min(i0 + 1, nT - 1);
    return lerp_at(col, i0, i1, coord_frac<R>(q));
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

// Band index of a uniform u on a cumulative table: the first b with
// u < cdf[b], with the reference's edge rules (R < cdf[0] -> 0, R == 1 ->
// n-1, mc_gpu_noint.cu:1113-1127).  For a non-decreasing cdf this is the
// same index the reference's bisection returns; the guide table gives the
// first band with cdf > q/kGuide, from which a short linear scan finishes.
template <typename R>
__device__ __forceinline__ int guided_index(const R *cdf, const int *guide, int n, R u) {
    const int q = min((int)(u * (R)kGuide), kGuide - 1);
    int b = guide[q];
    while (b < n - 1 && !(u < cdf[b])) ++b;
    return u == (R)1 ? n - 1 : b;
}

// Band and g point of an emitted bundle from its two uniforms: fluid bundles
// (kind 0) search the band CDF at the table row nearest Tmax and then the
// g CDF of that band and row (find_band, mc_gpu_noint.cu:1103-1169); wall
// bundles (kind 1, 2) the Planck-only wall band CDF and the constant g CDF
// probq (find_bandS :1170-1233, with the wall CDF's own edge rule).
template <typename R>
__device__ __forceinline__ void select_band_g(const DSolve<R> &S, int kind, R u_b, R u_g, int &nb, int &g) {
    if (kind == 0) {
        nb = (int)RC_IX(guided_index(S.cdf_f, S.guide_f, S.nB, u_b), S.nB, SITE_CDF, S);
        g = (S.nQ > 1)
                ? bisect(S.probg + RC_IX(((size_t)S.row * S.nB + nb) * S.nQ, (long long)S.nT * S.nB * S.nQ,
                                         SITE_PROBG, S),
                         S.nQ, u_g)
                : 0;
    } else {
        nb = (int)RC_IX(guided_index(S.cdf_s, S.guide_s, S.nB, u_b), S.nB, SITE_CDF, S);
        g = (S.nQ > 1) ? bisect(S.probq, S.nQ, u_g) : 0;
    }
}

// A bundle after emission, placed at its start point: position, cell,
// direction, sampled band/g and OERM weights.
template <typename R>
struct alignas(16) Emitted {
    R sx, sy, sz, ratioI, invTi4;
    int ij;    // ic | jc << 16: the emitting cell (fluid) or wall cell
    int kk;    // kc | kind << 16 | pool index << 18 | pool parity << 29
    int nbg;   // nb | g << 20
};

template <typename R>
struct Ray {
    R xp, yp, zp;
    R sx, sy, sz;
    R isx, isy, isz;
    R tra;
    R Ibmax, ratioI, invTi4, tol;
    const KIRow<R> *kicol;
    int ic, jc, kc;
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

// Emission of one bundle, placed at its start point.  kind 0: fluid cell
// (i,j,k) from its centre (kernel_fluid :115-186); kind 1/2: west/east wall
// cell (j,k) from the wall (kernel_surface :1381-1441).  Returns false if
// the bundle carries no energy.
//
// OERM weights: invTi4 = 1/I_b(Ti); ratioI = (I_b(Ti) k(Ti)) / (I_b(Tmax)
// k(Tmax)) for the fluid (the reference's ((1/invTi4)/Ib(Tmax))*k(Ti)/
// k(Tmax), :180-186) and I_b(Ti)/I_b(Tmax) for walls (:1421-1424).
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
    int Pi;
    int nb, g, ic = i;
    R st;
    if (kind == 0) {
        // isotropic: cos(theta) = 1 - 2u (emiss_ang, :1077-1084)
        const R mu = (R)1 - (R)2 * u_mu;
        st = RT<R>::sqrt_(((R)1 - mu) * ((R)1 + mu));
        e.sx = mu;
        select_band_g(S, 0, u_b, u_g, nb, g);
        const DLevel<R> &L0 = S.lev[0];
        Pi = L0.P[RC_IX(cell_index(i, j, k, L0.im, L0.jm), (long long)L0.im * L0.jm * L0.km, SITE_EMIT_T, S)];
    } else {
        // Lambertian: theta = acos(1 - 2u)/2 (+pi/2 on the east wall)
        // (emiss_angS, :1093-1102), i.e. cos = sqrt(1-u) / -sqrt(u).
        const int bound = kind - 1;
        if (bound == 0) {
            e.sx = RT<R>::sqrt_((R)1 - u_mu);
            st = RT<R>::sqrt_(u_mu);
        } else {
            e.sx = -RT<R>::sqrt_(u_mu);
            st = RT<R>::sqrt_((R)1 - u_mu);
        }
        select_band_g(S, kind, u_b, u_g, nb, g);
        Pi = S.Pw0[bound][RC_IX((k - 1) * S.jmax + (j - 1), (long long)S.kmax * S.jmax, SITE_WALL_EMIT_T, S)];
        ic = (bound == 0) ? 1 : S.imax;
    }
    e.sy = st * cp;
    e.sz = st * sp;
    if (kind == 0) {
        if (e.sx == (R)0) e.sx = (R)1e-10;  // :132-137
        if (e.sy == (R)0) e.sy = (R)1e-10;
        if (e.sz == (R)0) e.sz = (R)1e-10;
    } else {
        const int bound = kind - 1;
        if (RT<R>::fabs_(e.sx) <= (R)1e-10) e.sx = (R)(1 - 2 * bound) * (R)1e-10;  // :1395-1400
        if (RT<R>::fabs_(e.sy) <= (R)1e-10) e.sy = (R)((e.sy > (R)0) - (e.sy <= (R)0)) * (R)1e-10;
        if (RT<R>::fabs_(e.sz) <= (R)1e-10) e.sz = (R)((e.sz > (R)0) - (e.sz <= (R)0)) * (R)1e-10;
    }
    e.nbg = nb | (g << 20);
    e.ij = ic | (j << 16);
    e.kk = k | (kind << 16);
    // OERM weights
    const KIRow<R> row =
        S.ki[RC_IX(((size_t)nb * S.nQ + g) * S.nT + (Pi >> 8), (long long)S.nB * S.nQ * S.nT, SITE_EMIT_ROW, S)];
    const R fr = coord_frac<R>(Pi);
    const R Ib_i = RT<R>::lerp_(row.ib0, row.ib1, fr);
    if (!(Ib_i > (R)0)) return false;
    e.invTi4 = (R)1 / Ib_i;
    if (kind == 0) {
        const R k_i = RT<R>::lerp_(row.k0, row.k1, fr);
        const R den = S.den_f[RC_IX((size_t)nb * S.nQ + g, (long long)S.nB * S.nQ, SITE_DEN, S)];
        if (!(den > (R)0)) return false;
        e.ratioI = (Ib_i * k_i) / den;
    } else {
        const R den = S.ibm[RC_IX(nb, S.nB, SITE_IBM, S)];
        if (!(den > (R)0)) return false;
        e.ratioI = Ib_i / den;
    }
    return true;
}

// Ray state of an emitted bundle.
template <typename R>
__device__ __forceinline__ void place_bundle(Ray<R> &r, const DSolve<R> &S, const Emitted<R> &e) {
    const int kind = (e.kk >> 16) & 3;
    int ic = e.ij & 0xffff, jc = e.ij >> 16, kc = e.kk & 0xffff;
    // start point: the cell centre, or the wall cell's point on the wall
    // (kernel_fluid :117-122, kernel_surface :1381-1384)
    r.xp = kind == 0 ? S.xc[RC_IX(ic, S.imax + 2, SITE_CENTRE, S)] : (kind == 1 ? (R)0 : S.Lx);
    r.yp = S.yc[RC_IX(jc, S.jmax + 2, SITE_CENTRE, S)];
    r.zp = S.zc[RC_IX(kc, S.kmax + 2, SITE_CENTRE, S)];
    if (kind != 0) {
        // cell shift when the start point lies on a face (:1429-1441)
        const DLevel<R> &G = S.lev[0];
        const bool fx = e.sx < (R)0, fy = e.sy < (R)0, fz = e.sz < (R)0;
        const int i0 = ic, j0 = jc, k0 = kc;
        if (fx && r.xp == G.xu[RC_IX(i0 - 1, G.im + 1, SITE_FACE_SHIFT, S)]) ic = i0 - 1;
        if (fy && r.yp == G.yu[RC_IX(j0 - 1, G.jm + 1, SITE_FACE_SHIFT, S)]) jc = j0 - 1;
        if (fz && r.zp == G.zu[RC_IX(k0 - 1, G.km + 1, SITE_FACE_SHIFT, S)]) kc = k0 - 1;
        if (!fx && r.xp == G.xu[RC_IX(ic, G.im + 1, SITE_FACE_SHIFT, S)]) ic = ic + 1;
        if (!fy && r.yp == G.yu[RC_IX(jc, G.jm + 1, SITE_FACE_SHIFT, S)]) jc = jc + 1;
        if (!fz && r.zp == G.zu[RC_IX(kc, G.km + 1, SITE_FACE_SHIFT, S)]) kc = kc + 1;
    }
    r.sx = e.sx;
    r.sy = e.sy;
    r.sz = e.sz;
    r.isx = (R)1 / e.sx;
    r.isy = (R)1 / e.sy;
    r.isz = (R)1 / e.sz;
    r.ratioI = e.ratioI;
    r.invTi4 = e.invTi4;
    const int nb = e.nbg & 0xfffff, g = e.nbg >> 20;
    r.nb = nb;
    r.kicol = S.ki + ((size_t)nb * S.nQ + g) * S.nT;
    r.ic = ic;
    r.jc = jc;
    r.kc = kc;
    r.lev = 0;
    r.counter = 0;
    r.tra = (R)1;
    r.De = 0.0;
    r.Ibmax = kind == 0 ? S.Ibmax_f : kind == 1 ? S.Ibmax_w0 : S.Ibmax_w1;
    r.tol = kind == 0 ? S.toll : S.tollS;
}

// Deposit the remaining energy on a black wall emitting Ib_wall
// (:398-399 and its siblings): De -= Ibmax*tra*(invTi4*e - 1)*ratioI.
template <typename R>
__device__ __forceinline__ void wall_deposit(Ray<R> &r, R e) {
    R c = (r.Ibmax * r.tra) * RT<R>::fma_(r.invTi4, e, (R)-1);
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
        wall_deposit(r, S.Ibw[RC_IX((size_t)w * S.nB + r.nb, 6LL * S.nB, SITE_IBW, S)]);
    } else if (t == 4 || t == 6) {  // black wall at a field temperature
        int idx;
        if (w <= RC_EAST) idx = (r.kc - 1) * L.jm + (r.jc - 1);
        else if (w <= RC_NORTH) idx = (r.kc - 1) * L.im + (r.ic - 1);
        else idx = (r.jc - 1) * L.im + (r.ic - 1);
        const int q = L.Pw[w][RC_IX(idx, w <= RC_EAST ? (long long)L.jm * L.km : (w <= RC_NORTH ? (long long)L.im * L.km
                                                                                              : (long long)L.im * L.jm),
                                    SITE_WALL_T, S)];
        const KIRow<R> row = r.kicol[RC_IX(q >> 8, S.nT, SITE_WALL_ROW, S)];
        const R fr = coord_frac<R>(q);
        wall_deposit(r, RT<R>::lerp_(row.ib0, row.ib1, fr));
    } else if (t == 3) {  // specular
        switch (w) {
            case RC_WEST: r.xp = (R)0; r.sx = -r.sx; r.isx = -r.isx; r.ic = 1; break;
            case RC_EAST: r.xp = S.Lx; r.sx = -r.sx; r.isx = -r.isx; r.ic = L.im; break;
            case RC_SOUTH: r.yp = (R)0; r.sy = -r.sy; r.isy = -r.isy; r.jc = 1; break;
            case RC_NORTH: r.yp = S.Ly; r.sy = -r.sy; r.isy = -r.isy; r.jc = L.jm; break;
            case RC_BOT: r.zp = (R)0; r.sz = -r.sz; r.isz = -r.isz; r.kc = 1; break;
            default: r.zp = S.Lz; r.sz = -r.sz; r.isz = -r.isz; r.kc = L.km; break;
        }
    } else {  // lost ray
        r.tra = (R)0;
    }
}

// Absorption along a path of length ds in a cell of absorption coefficient
// absco and blackbody intensity blackpow: the step's OERM tally, the
// transmissivity update and the cutoff deposit (:358-370).
template <typename R>
__device__ __forceinline__ void absorb(Ray<R> &r, R ds, R absco, R blackpow) {
    const R em = RT<R>::expm1_(-(ds * absco));
    const R alpha = -em;
    const R dI = RT<R>::fma_(r.invTi4, blackpow, (R)-1);
    R c = r.Ibmax * r.tra;
    c = c * alpha;
    c = c * r.ratioI;
    c = c * dI;
    r.De -= (double)c;
    r.tra = RT<R>::fma_(r.tra, em, r.tra);
    if (r.tra < r.tol) {  // cutoff: deposit the rest here (:365-370)
        R c2 = (r.Ibmax * r.tra) * r.ratioI;
        c2 = c2 * dI;
        r.De -= (double)c2;
        r.tra = (R)0;
    }
}

// ---------------------------------------------------------------------------
// scattering by suspended particles
// ---------------------------------------------------------------------------
// The reference's Monte Carlo path has no scattering; nbcorrk tabulates the
// particles' scattering coefficient per band and g point and their phase
// function per band (nbcorrk/write_tables.cpp:204-260, :326-336).  A bundle
// of a scattering medium carries, besides its Ray, the Philox counter words
// of its emission (h, v | kind << 24, cell): draw n (the fourth counter word
// n >= 1; emission uses 0) is its n-th draw after emission.  Draw 1 gives
// the free path to the first scattering event, -ln(u) / k_s with k_s the
// scattering coefficient of its band and g point (no event when k_s = 0);
// at event n draw n+1 gives the scattering angle (the band's cumulative
// phase probability inverted, linear in angle between table angles), the
// azimuth (uniform) and the free path to the next event.  The free path is
// sampled against the scattering coefficient alone; absorption stays the
// continuous OERM tally, so the emission-based reciprocity weights are
// unchanged (the exchange between two cells is reciprocal for a phase
// function of the scattering angle alone).
// What a step needs of a scattering bundle is one register: the distance
// left to its next event.  The counter words, event count and k_s (needed
// only at an event) are kept apart, in shared memory in the march.
constexpr float kNoEvent = 3.0e38f;  // free path of a bundle whose band does not scatter
template <typename R>
struct ScatState {
    R dist;  // distance left to the next event; < 0: stopped at an event,
             // new direction not drawn yet
};

// Scattering coefficient of band nb, g point g (0 without particles).
template <typename R>
__device__ __forceinline__ R scatter_coef(const DSolve<R> &S, int nb, int g) {
    return (S.nA > 0) ? S.ksca[RC_IX((size_t)nb * S.nQ + g, (long long)S.nB * S.nQ, SITE_KSCA, S)] : (R)0;
}

// Philox counter words of a bundle (emission's: h, v | kind << 24, cell),
// with the event count in w.
__device__ __forceinline__ uint4 scatter_counter(uint32_t imax, uint32_t jmax, int kind, int i, int j, int k, int v,
                                                 int h, uint32_t nev) {
    const uint32_t cell = (kind == 0) ? (uint32_t)((i - 1) + imax * ((j - 1) + jmax * (k - 1)))
                                      : (uint32_t)((j - 1) + jmax * (k - 1));
    return make_uint4((uint32_t)h, (uint32_t)v | ((uint32_t)kind << 24), cell, nev);
}

// -ln(u) of draw 1 of a bundle with counter words ctr: its free path to the
// first event in units of 1/k_s.  The draw does not depend on the band, so
// the march takes it before the band is sampled (what is live at that
// point is small).
template <typename R>
__device__ __forceinline__ R scatter_first_lnu(const DSolve<R> &S, uint4 ctr) {
    rc_u32x4 c;
    c.x = ctr.x;
    c.y = ctr.y;
    c.z = ctr.z;
    c.w = 1u;
    const rc_u32x4 d = rc_philox4x32_10(c, S.key0, S.key1);
    return -RT<R>::log_((R)rc_u01(d.x));
}

// Free path to the first event: lnu / ks, kNoEvent when ks = 0.
template <typename R>
__device__ __forceinline__ R scatter_first_dist(R lnu, R ks) {
    return (ks > (R)0) ? lnu / ks : (R)kNoEvent;
}

// Angle index of a uniform u on the phase CDF of a band: the first a in
// [1, nA-1] with u < cdf[a] (nA-1 if none), which is what a bisection over
// the whole table returns for a CDF that starts at 0 and does not decrease.
// guide[q] (q = 0..kPhaseGuide) is the first a >= 1 with cdf[a] > q /
// kPhaseGuide (nA-1 if none), so for u in bucket q the answer lies in
// (guide[q] - 1, guide[q+1]] and the bisection runs over that bracket only:
// one or two table reads instead of log2(nA) dependent ones.
template <typename R>
__device__ __forceinline__ int phase_index(const R *cdf, const uint16_t *guide, R u) {
    const int q = min((int)(u * (R)kPhaseGuide), kPhaseGuide - 1);
    int lo = (int)guide[q] - 1, hi = (int)guide[q + 1];
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (u < cdf[mid]) hi = mid;
        else lo = mid;
    }
    return hi;
}

// New direction of a bundle travelling along (sx, sy, sz) in band nb at a
// scattering event (ctr: its counter words x, y, z and the number of the
// event in w; ks > 0 its scattering coefficient), with the reciprocals of
// the new direction and the free path to the event after it.  Everything is
// passed and returned by value: a reference would oblige the caller to keep
// the ray in local memory.
template <typename R>
struct TurnOut {
    R sx, sy, sz, isx, isy, isz, dist;
};
template <typename R>
__device__ __forceinline__ TurnOut<R> scatter_turn_v(R sx, R sy, R sz, int nb, uint4 ctr, R ks, const DSolve<R> *Sp) {
    const DSolve<R> &S = *Sp;
    rc_u32x4 c;
    c.x = ctr.x;
    c.y = ctr.y;
    c.z = ctr.z;
    c.w = ctr.w + 1u;
    const rc_u32x4 d = rc_philox4x32_10(c, S.key0, S.key1);
    const R u_t = (R)rc_u01(d.x), u_p = (R)rc_u01(d.y), u_s = (R)rc_u01(d.z);
    const int nA = S.nA;
    const R *cdf = S.pcdf + RC_IX((size_t)nb * nA, (long long)S.nB * nA, SITE_PHASE, S);
    const int hi = phase_index(cdf, S.pguide + RC_IX((size_t)nb * (kPhaseGuide + 1),
                                                     (long long)S.nB * (kPhaseGuide + 1), SITE_PHASE, S), u_t);
    const R c0 = cdf[hi - 1], c1 = cdf[hi];
    R fr = (c1 > c0) ? (u_t - c0) / (c1 - c0) : (R)0;
    if (fr > (R)1) fr = (R)1;
    const R t0 = S.pth[hi - 1], t1 = S.pth[hi];
    const R th = RT<R>::fma_(fr, t1 - t0, t0);
    R st, ct, sp, cp;
    RT<R>::sincos2pi_(th, &st, &ct);
    RT<R>::sincos2pi_(u_p, &sp, &cp);
    R nx, ny, nz;
    if (RT<R>::fabs_(sz) > (R)0.99999) {
        nx = st * cp;
        ny = st * sp;
        nz = (sz > (R)0) ? ct : -ct;
    } else {
        const R w = RT<R>::sqrt_((R)1 - sz * sz);
        const R a = st / w;
        nx = a * (sx * sz * cp - sy * sp) + sx * ct;
        ny = a * (sy * sz * cp + sx * sp) + sy * ct;
        nz = sz * ct - st * cp * w;
    }
    if (nx == (R)0) nx = (R)1e-10;
    if (ny == (R)0) ny = (R)1e-10;
    if (nz == (R)0) nz = (R)1e-10;
    TurnOut<R> o;
    o.sx = nx;
    o.sy = ny;
    o.sz = nz;
    o.isx = (R)1 / nx;
    o.isy = (R)1 / ny;
    o.isz = (R)1 / nz;
    o.dist = -RT<R>::log_(u_s) / ks;
    return o;
}

// The next scattering event of ray r: the event count in ctr.w advances,
// the direction turns, and q receives the free path to the event after it.
template <typename R>
__device__ __forceinline__ void scatter_turn(Ray<R> &r, uint4 &ctr, R ks, ScatState<R> &q, const DSolve<R> &S) {
    ctr.w += 1u;
    const TurnOut<R> o = scatter_turn_v(r.sx, r.sy, r.sz, r.nb, ctr, ks, &S);
    r.sx = o.sx;
    r.sy = o.sy;
    r.sz = o.sz;
    r.isx = o.isx;
    r.isy = o.isy;
    r.isz = o.isz;
    q.dist = o.dist;
}

// One ray-cell crossing (one iteration of the while loop of march_ray,
// :252-656).  Returns the step budget (maxs) of the level the step was
// taken on, which the caller compares with the step counter.  The side of
// the cell a ray leaves through on each axis follows from the sign of its
// direction component (never 0: emission floors it at 1e-10).  With SCAT, a
// bundle whose step is longer than the distance left to its next event
// stops at the event inside the cell (absorbing along the shortened path),
// counts the event as a step and sets qs.dist < 0: the caller draws the new
// direction (scatter_turn) before the next step.  The
// turn depends neither on the cell nor on the level, so a caller may
// advance the level first and gather the turns of several lanes into one
// pass.
template <typename R, bool SCAT>
__device__ __forceinline__ int march_step(Ray<R> &r, ScatState<R> &qs, const DSolve<R> &S) {
    // S lives in global memory (read-only during every kernel that steps)
    const int4 A = __ldg(&S.lva[RC_IX(r.lev, S.nlev, SITE_LEVEL, S)]);
    const int4 B = __ldg(&S.lvb[RC_IX(r.lev, S.nlev, SITE_LEVEL, S)]);
    const R fxu = __ldg(S.faces + RC_IX(A.x + r.ic - (int)(r.sx < (R)0), S.n_faces, SITE_FACE, S));
    const R fyu = __ldg(S.faces + RC_IX(A.y + r.jc - (int)(r.sy < (R)0), S.n_faces, SITE_FACE, S));
    const R fzu = __ldg(S.faces + RC_IX(A.z + r.kc - (int)(r.sz < (R)0), S.n_faces, SITE_FACE, S));
#if RC_CHECKED
    // the cell itself must lie inside its level (a face index alone can be
    // in the shared faces array while the cell is off its level)
    if (r.ic < 1 || r.ic > B.x || r.jc < 1 || r.jc > B.y || r.kc < 1 || r.kc > B.z) RC_IX(-1, 0, SITE_PYRAMID, S);
#endif
    const int q = __ldg(S.Pall + RC_IX(A.w + cell_index(r.ic, r.jc, r.kc, B.x, B.y), S.n_P, SITE_PYRAMID, S));
    const KIRow<R> row = load_row(r.kicol + RC_IX(q >> 8, S.nT, SITE_ROW, S));
    const R dsx = (fxu - r.xp) * r.isx;
    const R dsy = (fyu - r.yp) * r.isy;
    const R dsz = (fzu - r.zp) * r.isz;
    const R a = coord_frac<R>(q);
    const R absco = RT<R>::lerp_(row.k0, row.k1, a);
    const R blackpow = RT<R>::lerp_(row.ib0, row.ib1, a);
    R ds = dsx;
    if (ds > dsy) ds = dsy;
    if (ds > dsz) ds = dsz;
    // with SCAT, ev: the next scattering event lies inside this cell; the
    // bundle stops there (one absorption path shared with the plain step,
    // so the step loop's code does not grow)
    R dstep = ds;
    bool ev = false;
    if constexpr (SCAT) {
        ev = ds > qs.dist;
        dstep = ev ? qs.dist : ds;
        qs.dist = ev ? (R)-1 : qs.dist - ds;
    }
    r.xp = (!ev && ds == dsx) ? fxu : RT<R>::fma_(dstep, r.sx, r.xp);
    r.yp = (!ev && ds == dsy) ? fyu : RT<R>::fma_(dstep, r.sy, r.yp);
    r.zp = (!ev && ds == dsz) ? fzu : RT<R>::fma_(dstep, r.sz, r.zp);
    absorb(r, dstep, absco, blackpow);
    if constexpr (SCAT) {
        if (ev) {
            r.counter += 1;
            return B.w;
        }
    }
    // crossed axis (ties: x only if strictly smallest, :375-377, 524)
    const int axis = (dsx < dsy) ? ((dsx < dsz) ? 0 : 2) : ((dsy < dsz) ? 1 : 2);
    const bool ax0 = axis == 0, ax1 = axis == 1;
    const bool f = ax0 ? (r.sx < (R)0) : (ax1 ? (r.sy < (R)0) : (r.sz < (R)0));
    const int dlt = f ? -1 : 1;
    r.ic += ax0 ? dlt : 0;
    r.jc += ax1 ? dlt : 0;
    r.kc += (axis == 2) ? dlt : 0;
    const int nidx = ax0 ? r.ic : (ax1 ? r.jc : r.kc);
    const int lim = (ax0 ? B.x : (ax1 ? B.y : B.z)) + 1;
    if (nidx == 0 || nidx == lim) {
        const int w = 2 * axis + (nidx != 0);
        if (S.wtype[w] == 1) {
            // periodic (the common wall of the channel): re-enter through the
            // opposite face, on a short path of its own
            const bool hi = nidx != 0;
            const int ni = hi ? 1 : lim - 1;
            if (axis == 0) {
                r.ic = ni;
                r.xp = hi ? (R)0 : S.Lx;
            } else if (axis == 1) {
                r.jc = ni;
                r.yp = hi ? (R)0 : S.Ly;
            } else {
                r.kc = ni;
                r.zp = hi ? (R)0 : S.Lz;
            }
        } else {
            hit_wall(r, S, S.lev[r.lev], w);
        }
    }
    r.counter += 1;
    return B.w;
}

// Index of the coarse cell holding fine cell n (1-based): (n + r - 1) / r,
// as floor(n' m / 2^32) with m = floor(2^32 / r) + 1, exact for n' r < 2^32
// (the host checks it); m = 0 stands for r = 1.
__device__ __forceinline__ int coarse_index(int n, int r, unsigned m) {
    const unsigned np = (unsigned)(n + r - 1);
    return (int)(m ? __umulhi(np, m) : np);
}

// Advance to coarser levels while the step budget of the current level is
// spent (:210-224).  Returns false when the ray must stop (budget of the
// last level spent).
template <typename R>
__device__ __forceinline__ bool level_advance(Ray<R> &r, const DSolve<R> &S) {
    while (r.counter >= __ldg(&S.lvb[r.lev]).w) {
        if (r.lev >= S.nlev - 1) return false;
        const DLevel<R> &L = S.lev[r.lev];
        r.ic = coarse_index(r.ic, L.rx, L.mrx);
        r.jc = coarse_index(r.jc, L.ry, L.mry);
        r.kc = coarse_index(r.kc, L.rz, L.mrz);
        r.lev += 1;
        r.counter = 0;
    }
    return true;
}

// n / d for a divisor fixed per solve: with M = floor((2^64 - 1)/d) + 1,
// floor(n M / 2^64) = floor(n / d) whenever n d < 2^64 (the host checks the
// bound when it builds the descriptor); M = 0 encodes d = 1.
__device__ __forceinline__ unsigned long long fdiv(unsigned long long n, unsigned long long M) {
    return M ? __umul64hi(n, M) : n;
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
    unsigned long long it = (unsigned long long)item;
    int kind = 0;
    if (item >= S.n_fluid_items) {
        it -= (unsigned long long)S.n_fluid_items;
        kind = 1;
    }
    const unsigned long long t = fdiv(it, S.mg_nchunk);
    const int q = (int)(it - t * (unsigned long long)S.nchunk);
    const unsigned long long c = fdiv(t, S.mg_nvar);
    d.v = (int)(t - c * (unsigned long long)S.nVar);
    d.h0 = q * S.rpt;
    if (kind == 0) {
        const unsigned long long cj = fdiv(c, S.mg_imax);
        d.i = (int)(c - cj * (unsigned long long)S.imax) + 1;
        const unsigned long long ck = fdiv(cj, S.mg_jmax);
        d.j = (int)(cj - ck * (unsigned long long)S.jmax) + 1;
        d.k = (int)ck + S.kfirst;
        d.kind = 0;
    } else {
        const unsigned long long slot = fdiv(c, S.mg_nwc);
        const unsigned long long wc = c - slot * S.nwc;
        const unsigned long long kw = fdiv(wc, S.mg_jmax);
        d.j = (int)(wc - kw * (unsigned long long)S.jmax) + 1;
        d.k = (int)kw + S.kfirst;
        d.kind = 1 + S.wall_id[(int)slot];
    }
    return d;
}

}  // namespace rc
