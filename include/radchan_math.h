/*
 * radchan_math.h -- arithmetic primitives shared by the sm_100a kernels and
 * by host code (table builders, the CPU oracle).
 *
 * Every function here is written so that the host build (g++ with
 * -ffp-contract=off, no fast-math) and the device build (nvcc with
 * -fmad=false, IEEE division and square root) produce bit-identical results:
 * only IEEE add/mul/div/sqrt, explicit fmaf()/fma() (correctly rounded on
 * both sides), rintf()/rint() in round-to-nearest-even, and exact
 * power-of-two scaling through the exponent bits are used.
 *
 * Contents
 *  - Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 *    "Parallel random numbers: as easy as 1, 2, 3", SC'11).  Replaces the
 *    reference's cuRAND XORWOW/Sobol32 states (src/montecarlo/mc_gpu_noint.cu:83-87),
 *    whose per-thread seeds were not unique.
 *  - rc_u01(): 24-bit uniform on (0,1], the same open/closed interval as
 *    curand_uniform(), so the reference's "R == 1" edge rules stay meaningful.
 *  - rc_expf/rc_expm1f (and double versions): Cody-Waite argument reduction
 *    x = n*ln2 + r with ln2 split into a short high part and a low part,
 *    followed by the Taylor series of e^r (coefficients 1/k!) evaluated with
 *    Horner's rule.  Used for the absorption alpha = 1 - exp(-k ds)
 *    (mc_gpu_noint.cu:358, where the reference uses __expf).
 *  - rc_sincos2pif: sin/cos of 2*pi*u by reduction to the nearest quarter
 *    turn and Taylor series on [-pi/4, pi/4].  Used for the azimuth of
 *    emitted bundles (mc_gpu_noint.cu:1079-1083).
 *  - rc_logf/rc_log: natural logarithm by exponent extraction and the
 *    atanh series 2 (s + s^3/3 + s^5/5 + ...), s = (m-1)/(m+1).  Used for the
 *    free path -ln(u) between scattering events (optional particle media).
 *  - rc_planck: spectral blackbody intensity I_b(T, nu) with nu in cm^-1,
 *    restating I_blackC (src/montecarlo/memory_copy_noint.cu:288-297) in
 *    double precision with expm1 for the denominator.
 */
#ifndef RADCHAN_MATH_H_
#define RADCHAN_MATH_H_

#include <stdint.h>
#if defined(__CUDACC__)
#define RC_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define RC_HD static inline
#endif

/* ------------------------------------------------------------------ */
/* bit casts                                                           */
/* ------------------------------------------------------------------ */
RC_HD float rc_u32_as_f32(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}
RC_HD uint32_t rc_f32_as_u32(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
RC_HD double rc_u64_as_f64(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d; memcpy(&d, &u, 8); return d;
#endif
}
RC_HD uint64_t rc_f64_as_u64(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u; memcpy(&u, &d, 8); return u;
#endif
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10                                                       */
/* ------------------------------------------------------------------ */
#define RC_PHILOX_M0 0xD2511F53u
#define RC_PHILOX_M1 0xCD9E8D57u
#define RC_PHILOX_W0 0x9E3779B9u
#define RC_PHILOX_W1 0xBB67AE85u

typedef struct rc_u32x4 { uint32_t x, y, z, w; } rc_u32x4;

RC_HD void rc_mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
#if defined(__CUDA_ARCH__)
    *hi = __umulhi(a, b);
    *lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
#endif
}

/* One Philox4x32 bijection with 10 rounds; key schedule bumps (W0, W1)
 * between rounds. */
RC_HD rc_u32x4 rc_philox4x32_10(rc_u32x4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        rc_mulhilo32(RC_PHILOX_M0, c.x, &hi0, &lo0);
        rc_mulhilo32(RC_PHILOX_M1, c.z, &hi1, &lo1);
        rc_u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += RC_PHILOX_W0;
        k1 += RC_PHILOX_W1;
    }
    return c;
}

/* Uniform on (0, 1] with 24 random bits: ((x >> 8) + 1) * 2^-24.
 * Exactly representable in float and double. */
RC_HD float rc_u01(uint32_t x) {
    return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f;
}

/* ------------------------------------------------------------------ */
/* table interpolation                                                 */
/* ------------------------------------------------------------------ */
/* a0 (1 - w) + a1 w, the product a0 (1 - w) rounded and a1 w added in one
 * fused multiply-add (one rounding fewer than the plain expression, and
 * one instruction fewer on the device). */
RC_HD float rc_lerpf(float a0, float a1, float w) { return fmaf(a1, w, a0 * (1.0f - w)); }
RC_HD double rc_lerp(double a0, double a1, double w) { return fma(a1, w, a0 * (1.0 - w)); }

/* ------------------------------------------------------------------ */
/* exp / expm1, single precision                                       */
/* ------------------------------------------------------------------ */
/* ln2 = RC_LN2_HI_F + RC_LN2_LO_F; the high part keeps 16 significant bits
 * so n * RC_LN2_HI_F is exact for |n| <= 255. */
#define RC_LN2_HI_F  0.693145751953125f
#define RC_LN2_LO_F  1.428606765330187e-06f
#define RC_LOG2E_F   1.4426950216293335f

/* 2^n for integer n in [-126, 127], built from the exponent field. */
RC_HD float rc_exp2i_f(int n) {
    return rc_u32_as_f32((uint32_t)(n + 127) << 23);
}

/* e^r - 1 for |r| <= ~0.35: r * (1 + r/2! + r^2/3! + ... + r^6/7!); the
 * first omitted term, r^8/8!, is below 1.5e-8 relative (0.13 ulp). */
RC_HD float rc_expm1_poly_f(float r) {
    float p = 1.9841270113829523e-04f;          /* 1/7! */
    p = fmaf(p, r, 1.3888889225199819e-03f);    /* 1/6! */
    p = fmaf(p, r, 8.3333337679505348e-03f);    /* 1/5! */
    p = fmaf(p, r, 4.1666667908430099e-02f);    /* 1/4! */
    p = fmaf(p, r, 1.6666667163372040e-01f);    /* 1/3! */
    p = fmaf(p, r, 0.5f);                       /* 1/2! */
    p = fmaf(p, r, 1.0f);                       /* 1/1! */
    return r * p;
}

/* e^x.  Inputs below -87 return 0 (the caller only ever needs e^-tau with
 * tau >= 0, where such values are far below any transmissivity cutoff);
 * inputs above 88 return +inf. NaN propagates. */
RC_HD float rc_expf(float x) {
    if (x < -87.0f) return 0.0f;
    if (x > 88.0f) return rc_u32_as_f32(0x7f800000u);
    float n = rintf(x * RC_LOG2E_F);
    float r = fmaf(-n, RC_LN2_LO_F, fmaf(-n, RC_LN2_HI_F, x));
    float p = rc_expm1_poly_f(r) + 1.0f;
    return p * rc_exp2i_f((int)n);
}

/* e^x - 1 without cancellation near 0, branch-free:
 * e^x - 1 = 2^n (e^r - 1) + (2^n - 1), evaluated as one fused multiply-add.
 * For |x| < ln2/2, n = 0 and the result is the polynomial itself.
 * Arguments are clamped to [-87, 88] (e^-87 - 1 rounds to -1). */
RC_HD float rc_expm1f(float x) {
    x = fminf(fmaxf(x, -87.0f), 88.0f);
    float n = rintf(x * RC_LOG2E_F);
    /* n * ln2_hi is exact, so the inner fma is the exact x - n ln2_hi */
    float r = fmaf(-n, RC_LN2_LO_F, fmaf(-n, RC_LN2_HI_F, x));
    float p = rc_expm1_poly_f(r);
    float s = rc_exp2i_f((int)n);
    return fmaf(s, p, s - 1.0f);
}

/* ------------------------------------------------------------------ */
/* exp / expm1, double precision                                       */
/* ------------------------------------------------------------------ */
/* ln2 = RC_LN2_HI_D + RC_LN2_LO_D; the high part keeps 21 significant bits
 * so n * RC_LN2_HI_D is exact for |n| < 2^31. */
#define RC_LN2_HI_D  0.6931467056274414
#define RC_LN2_LO_D  4.7493250390316726e-07
#define RC_LOG2E_D   1.4426950408889634

RC_HD double rc_exp2i_d(int n) {
    return rc_u64_as_f64((uint64_t)(n + 1023) << 52);
}

/* e^r - 1 for |r| <= ~0.35, Taylor series through r^14/14! */
RC_HD double rc_expm1_poly_d(double r) {
    double p = 1.1470745597729725e-11;       /* 1/14! */
    p = fma(p, r, 1.6059043836821613e-10);   /* 1/13! */
    p = fma(p, r, 2.08767569878681e-09);     /* 1/12! */
    p = fma(p, r, 2.505210838544172e-08);    /* 1/11! */
    p = fma(p, r, 2.755731922398589e-07);    /* 1/10! */
    p = fma(p, r, 2.7557319223985893e-06);   /* 1/9!  */
    p = fma(p, r, 2.48015873015873e-05);     /* 1/8!  */
    p = fma(p, r, 1.984126984126984e-04);    /* 1/7!  */
    p = fma(p, r, 1.388888888888889e-03);    /* 1/6!  */
    p = fma(p, r, 8.333333333333333e-03);    /* 1/5!  */
    p = fma(p, r, 4.1666666666666664e-02);   /* 1/4!  */
    p = fma(p, r, 1.6666666666666666e-01);   /* 1/3!  */
    p = fma(p, r, 0.5);                      /* 1/2!  */
    p = fma(p, r, 1.0);                      /* 1/1!  */
    return r * p;
}

RC_HD double rc_exp(double x) {
    if (x < -708.0) return 0.0;
    if (x > 709.0) return rc_u64_as_f64(0x7ff0000000000000ull);
    double n = rint(x * RC_LOG2E_D);
    double r = (x - n * RC_LN2_HI_D) - n * RC_LN2_LO_D;
    double p = rc_expm1_poly_d(r) + 1.0;
    return p * rc_exp2i_d((int)n);
}

RC_HD double rc_expm1(double x) {
    x = fmin(fmax(x, -708.0), 709.0);
    double n = rint(x * RC_LOG2E_D);
    double r = (x - n * RC_LN2_HI_D) - n * RC_LN2_LO_D;
    double p = rc_expm1_poly_d(r);
    double s = rc_exp2i_d((int)n);
    return fma(s, p, s - 1.0);
}

/* ------------------------------------------------------------------ */
/* natural logarithm                                                   */
/* ------------------------------------------------------------------ */
/* ln x for finite x > 0 in the normal range: x = m 2^e with m in
 * [sqrt(1/2), sqrt(2)), ln x = e ln2 + 2 atanh(s) with s = (m-1)/(m+1),
 * |s| <= 0.1716, and atanh(s) = s + s^3/3 + s^5/5 + ... (the series in
 * powers of s^2, evaluated by Horner's rule).  m - 1 is exact (Sterbenz).
 * Used for the free path -ln(u) between scattering events. */
RC_HD float rc_logf(float x) {
    uint32_t b = rc_f32_as_u32(x);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = rc_u32_as_f32((b & 0x007fffffu) | 0x3f800000u);  /* [1, 2) */
    if (m > 1.41421354f) { m = m * 0.5f; e = e + 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    /* 2 atanh(s) = 2s (1 + s^2/3 + s^4/5 + s^6/7 + s^8/9); the first
     * omitted term, s^10/11, is below 5e-9 relative */
    float p = 1.1111111193895340e-01f;          /* 1/9 */
    p = fmaf(p, s2, 1.4285714924335480e-01f);   /* 1/7 */
    p = fmaf(p, s2, 2.0000000298023224e-01f);   /* 1/5 */
    p = fmaf(p, s2, 3.3333334326744080e-01f);   /* 1/3 */
    float t = 2.0f * s;
    float l = fmaf(t * s2, p, t);
    float fe = (float)e;
    return fmaf(fe, RC_LN2_HI_F, fmaf(fe, RC_LN2_LO_F, l));
}

RC_HD double rc_log(double x) {
    uint64_t b = rc_f64_as_u64(x);
    int e = (int)((b >> 52) & 0x7ffu) - 1023;
    double m = rc_u64_as_f64((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    /* 2s (1 + s^2/3 + ... + s^20/21); first omitted term s^22/23 < 6e-19 */
    double p = 4.7619047619047616e-02;        /* 1/21 */
    p = fma(p, s2, 5.2631578947368418e-02);   /* 1/19 */
    p = fma(p, s2, 5.8823529411764705e-02);   /* 1/17 */
    p = fma(p, s2, 6.6666666666666666e-02);   /* 1/15 */
    p = fma(p, s2, 7.6923076923076927e-02);   /* 1/13 */
    p = fma(p, s2, 9.0909090909090912e-02);   /* 1/11 */
    p = fma(p, s2, 1.1111111111111111e-01);   /* 1/9 */
    p = fma(p, s2, 1.4285714285714285e-01);   /* 1/7 */
    p = fma(p, s2, 2.0000000000000001e-01);   /* 1/5 */
    p = fma(p, s2, 3.3333333333333331e-01);   /* 1/3 */
    double t = 2.0 * s;
    double l = fma(t * s2, p, t);
    double fe = (double)e;
    return fma(fe, RC_LN2_HI_D, fma(fe, RC_LN2_LO_D, l));
}

/* ------------------------------------------------------------------ */
/* sin/cos of 2*pi*u                                                   */
/* ------------------------------------------------------------------ */
#define RC_TWO_PI_F 6.2831854820251465f
#define RC_TWO_PI_D 6.283185307179586

/* Taylor series of sin and cos on |r| <= pi/4 (error < 2e-9). */
RC_HD void rc_sincos_poly_f(float r, float *s, float *c) {
    float r2 = r * r;
    float ps = 2.7557318844628753e-06f;           /* 1/9! */
    ps = fmaf(ps, r2, -1.9841270113829523e-04f);  /* -1/7! */
    ps = fmaf(ps, r2, 8.3333337679505348e-03f);   /* 1/5! */
    ps = fmaf(ps, r2, -1.6666667163372040e-01f);  /* -1/3! */
    *s = fmaf(ps * r2, r, r);
    float pc = -2.7557319981497130e-07f;          /* -1/10! */
    pc = fmaf(pc, r2, 2.4801587642286904e-05f);   /* 1/8! */
    pc = fmaf(pc, r2, -1.3888889225199819e-03f);  /* -1/6! */
    pc = fmaf(pc, r2, 4.1666667908430099e-02f);   /* 1/4! */
    pc = fmaf(pc, r2, -0.5f);                     /* -1/2! */
    *c = fmaf(pc, r2, 1.0f);
}

/* (sin, cos) of 2*pi*u for u in [0, 1]: u = q/4 + f with |f| <= 1/8 exact,
 * angle 2*pi*f on [-pi/4, pi/4], then rotate by q quarter turns. */
RC_HD void rc_sincos2pif(float u, float *s, float *c) {
    float q = rintf(u * 4.0f);
    float f = u - q * 0.25f;
    float ss, cc;
    rc_sincos_poly_f(f * RC_TWO_PI_F, &ss, &cc);
    int iq = ((int)q) & 3;
    if (iq == 0)      { *s = ss;  *c = cc;  }
    else if (iq == 1) { *s = cc;  *c = -ss; }
    else if (iq == 2) { *s = -ss; *c = -cc; }
    else              { *s = -cc; *c = ss;  }
}

RC_HD void rc_sincos_poly_d(double r, double *s, double *c) {
    double r2 = r * r;
    double ps = -7.647163731819816e-13;         /* -1/15! */
    ps = fma(ps, r2, 1.6059043836821613e-10);   /* 1/13! */
    ps = fma(ps, r2, -2.505210838544172e-08);   /* -1/11! */
    ps = fma(ps, r2, 2.7557319223985893e-06);   /* 1/9! */
    ps = fma(ps, r2, -1.984126984126984e-04);   /* -1/7! */
    ps = fma(ps, r2, 8.333333333333333e-03);    /* 1/5! */
    ps = fma(ps, r2, -1.6666666666666666e-01);  /* -1/3! */
    *s = fma(ps * r2, r, r);
    double pc = 4.779477332387385e-14;          /* 1/16! */
    pc = fma(pc, r2, -1.1470745597729725e-11);  /* -1/14! */
    pc = fma(pc, r2, 2.08767569878681e-09);     /* 1/12! */
    pc = fma(pc, r2, -2.755731922398589e-07);   /* -1/10! */
    pc = fma(pc, r2, 2.48015873015873e-05);     /* 1/8! */
    pc = fma(pc, r2, -1.388888888888889e-03);   /* -1/6! */
    pc = fma(pc, r2, 4.1666666666666664e-02);   /* 1/4! */
    pc = fma(pc, r2, -0.5);                     /* -1/2! */
    *c = fma(pc, r2, 1.0);
}

RC_HD void rc_sincos2pi(double u, double *s, double *c) {
    double q = rint(u * 4.0);
    double f = u - q * 0.25;
    double ss, cc;
    rc_sincos_poly_d(f * RC_TWO_PI_D, &ss, &cc);
    int iq = ((int)q) & 3;
    if (iq == 0)      { *s = ss;  *c = cc;  }
    else if (iq == 1) { *s = cc;  *c = -ss; }
    else if (iq == 2) { *s = -ss; *c = -cc; }
    else              { *s = -cc; *c = ss;  }
}

/* ------------------------------------------------------------------ */
/* Planck function                                                     */
/* ------------------------------------------------------------------ */
/* First and second radiation constants exactly as the reference states
 * them (memory_copy_noint.cu:292-293): C1 = 2*pi*h*c^2 [W m^2],
 * C2 = h*c/k [m K]. */
#define RC_PLANCK_C1 3.741771790075259e-16
#define RC_PLANCK_C2 0.014387741858429
#define RC_PI_D      3.14159265358979323846

/* Spectral blackbody intensity per unit wavenumber (nu in cm^-1, result in
 * W / (m^2 sr m^-1)): C1 (100 nu)^3 / (pi (exp(C2 100 nu / T) - 1)).
 * T <= 0 (a cold wall, the reference's Tw = 0 default) gives 0. */
RC_HD double rc_planck(double T, double nu) {
    if (!(T > 0.0)) return 0.0;
    double eta = nu * 100.0;
    double x = RC_PLANCK_C2 * eta / T;
    if (x > 700.0) return 0.0;
    double den = rc_expm1(x);
    return RC_PLANCK_C1 * eta * eta * eta / (RC_PI_D * den);
}

/* ------------------------------------------------------------------ */
/* scattering table conversions (library and oracle alike)             */
/* ------------------------------------------------------------------ */
/* Scattering coefficient scaled by chanHeight as the reference scales k
 * on load (read_tables.cpp:30,56), rounded to float. */
RC_HD float rc_scatter_coef_scaled(float k, double chanHeight) {
    return (float)((double)k * chanHeight);
}
/* A scattering angle in radians as turns (theta / 2 pi), rounded to float:
 * the argument of rc_sincos2pif. */
RC_HD float rc_angle_turns(float theta) {
    return (float)((double)theta / (2.0 * RC_PI_D));
}

#endif /* RADCHAN_MATH_H_ */
