// rc_kernels.cuh -- kernels of one solve: set-up (Tmax, table rows, grey
// tables), multigrid temperature levels, the persistent march kernel and
// the tally.  Included once, by rc_solver.cu.
#pragma once
#include "rc_device.cuh"
#include "rc_march.cuh"

namespace rc {

// ---------------------------------------------------------------------------
// set-up
// ---------------------------------------------------------------------------

// Max of interior T and of the x-wall face averages (mc_gpu_noint.cu:696-710),
// min of interior T, and finiteness flags.
static __global__ void k_tmax(const float *__restrict__ T, int imax, int jmax, int kmax, DScalars *sc) {
    const long long n = (long long)imax * jmax * kmax;
    float mx = 0.f, mn = 3.4e38f;
    int st = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % imax) + 1;
        const long long r = c / imax;
        const int j = (int)(r % jmax) + 1;
        const int k = (int)(r / jmax) + 1;
        const long long base = (long long)(imax + 2) * (j + (long long)(jmax + 2) * k);
        const float v = T[base + i];
        if (!isfinite(v)) {
            st |= 2;
            continue;
        }
        if (v <= 0.f) st |= 4;
        mx = fmaxf(mx, v);
        mn = fminf(mn, v);
        if (i == 1) {
            const float f = (T[base] + T[base + 1]) * 0.5f;
            if (isfinite(f)) mx = fmaxf(mx, f);
            else st |= 2;
        }
        if (i == imax) {
            const float f = (T[base + imax] + T[base + imax + 1]) * 0.5f;
            if (isfinite(f)) mx = fmaxf(mx, f);
            else st |= 2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        st |= __shfl_xor_sync(0xffffffffu, st, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&sc->tmax_bits, __float_as_uint(fmaxf(mx, 0.f)));
        atomicMin(&sc->tmin_bits, __float_as_uint(fmaxf(mn, 0.f)));
        if (st) atomicOr(&sc->status, st);
    }
}

// Scalars of the solve (mc_gpu_noint.cu:74, 820-826, 1362-1366;
// read_tables.cpp:36-38, 102-110).  One warp.
template <typename R>
__global__ void k_setup1(DScalars *sc, R *Tnb, const R *kP, int nT, int grey, float Tmins, float abscoeff,
                         double stefan, int photmax, float eps_w, float eps_e) {
    const float Tmax_f = __uint_as_float(sc->tmax_bits);
    const R Tmax = (R)Tmax_f;
    if (grey) {
        for (int i = threadIdx.x; i < nT; i += blockDim.x)
            Tnb[i] = (R)((double)Tmins * 0.9 + ((double)Tmax * 1.1 - (double)Tmins * 0.9) * (double)(R)i / (double)(R)nT);
    }
    __syncwarp();
    if (threadIdx.x != 0) return;
    int status = sc->status;
    int tm = (int)((Tmax - Tnb[0]) / (Tnb[1] - Tnb[0]));
    if (tm < 0) {
        tm = 0;
        status |= 1;
    }
    if (tm > nT - 2) {
        tm = nT - 2;
        status |= 1;
    }
    const float Tmin_f = __uint_as_float(sc->tmin_bits);
    if ((R)Tmin_f < Tnb[0] || Tmax > Tnb[nT - 1]) status |= 1;
    const int row = ((Tmax - Tnb[tm]) < (Tnb[tm + 1] - Tmax)) ? tm : tm + 1;
    R kappamax;
    if (grey) kappamax = (R)abscoeff;
    else kappamax = (kP[tm + 1] - kP[tm]) / (Tnb[tm + 1] - Tnb[tm]) * (Tmax - Tnb[tm]) + kP[tm];
    const R T4 = Tmax * Tmax * Tmax * Tmax;
    const R kf = (R)4 * kappamax * T4;
    sc->tm = tm;
    sc->row = row;
    sc->status = status;
    sc->Tmax = (double)Tmax;
    sc->kappamax = (double)kappamax;
    sc->Ibmax_f = (double)(R)((double)kf * stefan / (double)photmax);
    sc->Ibmax_w[0] = (double)(R)((double)eps_w * stefan * (double)T4 / (double)photmax);
    sc->Ibmax_w[1] = (double)(R)((double)eps_e * stefan * (double)T4 / (double)photmax);
    const R T0 = Tnb[0];
    const R inv_dT = (R)1 / (Tnb[1] - Tnb[0]);
    sc->T0 = (double)T0;
    sc->inv_dT = (double)inv_dT;
    sc->Pm = table_coord(Tmax, T0, inv_dT, nT);
}

// Copy the run-time values of a solve into its descriptor (after k_setup1,
// before the march).
template <typename R>
__global__ void k_patch_desc(DSolve<R> *d, const DScalars *sc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        d->Pm = sc->Pm;
        d->Ibmax_f = (R)sc->Ibmax_f;
        d->Ibmax_w0 = (R)sc->Ibmax_w[0];
        d->Ibmax_w1 = (R)sc->Ibmax_w[1];
        d->row = sc->row;
    }
}

static __global__ void k_init_scalars(DScalars *sc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        DScalars z;
        memset(&z, 0, sizeof(z));
        z.tmax_bits = 0u;
        z.tmin_bits = 0x7f800000u;
        *sc = z;
    }
}

// Interleaved k / I_b rows {k[t], Ib[t], k[t+1], Ib[t+1]} (last row repeated).
template <typename R>
__global__ void k_build_ki(KIRow<R> *ki, const R *kt, const R *Ibt, int nB, int nQ, int nT) {
    const int n = nB * nQ * nT;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int t = e % nT, bg = e / nT, nb = bg / nQ;
        const int t1 = min(t + 1, nT - 1);
        KIRow<R> r;
        r.k0 = kt[(size_t)bg * nT + t];
        r.k1 = kt[(size_t)bg * nT + t1];
        r.ib0 = Ibt[(size_t)nb * nT + t];
        r.ib1 = Ibt[(size_t)nb * nT + t1];
        ki[e] = r;
    }
}

// Grey-gas Planck table I_b(Tnb[t], wvc[b]) (read_tables.cpp:140-148).
template <typename R>
__global__ void k_grey_ib(R *Ibt, const R *Tnb, const R *wvc, int nT, int nB) {
    const int n = nT * nB;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int b = e / nT, t = e % nT;
        Ibt[e] = (R)rc_planck((double)Tnb[t], (double)wvc[b]);
    }
}

// Cumulative Planck band probability of one table row
// (read_tables.cpp:153-165 grey, :204-218 walls).
template <typename R>
__device__ void planck_cdf_row(R *out, const R *Ibt, const R *wvl, const R *wvr, int nT, int nB, int row) {
    R c = Ibt[(size_t)0 * nT + row] * (wvr[0] - wvl[0]) * (R)100;
    out[0] = c;
    for (int b = 1; b < nB; ++b) {
        c = c + Ibt[(size_t)b * nT + row] * (wvr[b] - wvl[b]) * (R)100;
        out[b] = c;
    }
    const R last = out[nB - 1];
    for (int b = 0; b < nB; ++b) out[b] = out[b] / last;
}

// First index b with cdf[b] > x (n-1 if none).
template <typename R>
__device__ int first_above(const R *cdf, int n, R x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cdf[mid] > x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Per-solve sampling tables (one block): band CDF rows at the row nearest
// Tmax -- fluid (copy, or the grey Planck CDF) and walls (readS,
// read_tables.cpp:188-220) -- their guide tables, and the Tmax factors of
// the OERM weights, I_b(Tmax) k_g(Tmax) per (band, g) and I_b(Tmax) per band.
template <typename R>
__global__ void k_setup2(const DScalars *sc, R *cdf_f, R *cdf_s, int *guide_f, int *guide_s, R *den_f, R *ibm,
                         const R *prob, const R *Ibt, const R *kt, const R *wvl, const R *wvr, int nT, int nB,
                         int nQ, int grey, int walls) {
    const int row = sc->row;
    const int Pm = sc->Pm;
    if (!grey) {
        for (int b = threadIdx.x; b < nB; b += blockDim.x) cdf_f[b] = prob[(size_t)row * nB + b];
    }
    if (threadIdx.x == 0 && grey) planck_cdf_row(cdf_f, Ibt, wvl, wvr, nT, nB, row);
    if (threadIdx.x == 32 % blockDim.x && walls) planck_cdf_row(cdf_s, Ibt, wvl, wvr, nT, nB, row);
    for (int e = threadIdx.x; e < nB * nQ; e += blockDim.x) {
        const int nb = e / nQ, g = e % nQ;
        const R Ib_m = tab_lerp(Ibt + (size_t)nb * nT, nT, Pm);
        const R k_m = tab_lerp(kt + ((size_t)nb * nQ + g) * nT, nT, Pm);
        den_f[e] = Ib_m * k_m;
        if (g == 0) ibm[nb] = Ib_m;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kGuide; q += blockDim.x) {
        const R x = (R)q / (R)kGuide;
        guide_f[q] = first_above(cdf_f, nB, x);
        if (walls) guide_s[q] = first_above(cdf_s, nB, x);
    }
}

// Texture-space trilinear sample of the float field with clamped indices
// (the reference's tex3D with cudaFilterModeLinear/cudaAddressModeClamp,
// memory_copy_noint.cu:159-165), with exact float weights.
__device__ __forceinline__ float tex_sample(const float *T, int nx, int ny, int nz, float x, float y, float z) {
    const float xb = x - 0.5f, yb = y - 0.5f, zb = z - 0.5f;
    const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
    const float ax = xb - fx, ay = yb - fy, az = zb - fz;
    int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    i0 = min(max(i0, 0), nx - 1);
    i1 = min(max(i1, 0), nx - 1);
    j0 = min(max(j0, 0), ny - 1);
    j1 = min(max(j1, 0), ny - 1);
    k0 = min(max(k0, 0), nz - 1);
    k1 = min(max(k1, 0), nz - 1);
    auto at = [&](int i, int j, int k) { return T[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)]; };
    const float c00 = at(i0, j0, k0) * (1.f - ax) + at(i1, j0, k0) * ax;
    const float c10 = at(i0, j1, k0) * (1.f - ax) + at(i1, j1, k0) * ax;
    const float c01 = at(i0, j0, k1) * (1.f - ax) + at(i1, j0, k1) * ax;
    const float c11 = at(i0, j1, k1) * (1.f - ax) + at(i1, j1, k1) * ax;
    const float c0 = c00 * (1.f - ay) + c10 * ay;
    const float c1 = c01 * (1.f - ay) + c11 * ay;
    return c0 * (1.f - az) + c1 * az;
}

// One array of the multigrid temperature pyramid: the cell temperatures
// of a level (sampled at the coarse cell centre, mc_gpu_noint.cu:334-338)
// or the emission temperature of a wall at that level (:392-396, 468-472).
struct LevelJob {
    void *dst;
    int type;     // 0 cells, 1 + w: wall w
    int im, jm, km;
    int rx, ry, rz;   // fine cells per level cell (imax/im ...)
    int face;     // wall sampled at the face (1) or at the first cell (0)
    long long n, start;
};
constexpr int kMaxJobs = RC_MAX_LEVELS * 7 + 2;
struct LevelJobs {
    LevelJob job[kMaxJobs];
    int njobs;
    long long total;
};

template <typename R>
__global__ void k_levels(const float *__restrict__ T, int imax, int jmax, int kmax, LevelJobs jobs,
                         const DScalars *sc, int nT) {
    const int nx = imax + 2, ny = jmax + 2, nz = kmax + 2;
    const R T0 = (R)sc->T0, inv_dT = (R)sc->inv_dT;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < jobs.total;
         e += (long long)gridDim.x * blockDim.x) {
        int jb = 0;
        while (jb + 1 < jobs.njobs && jobs.job[jb + 1].start <= e) ++jb;
        const LevelJob &J = jobs.job[jb];
        const long long l = e - J.start;
        uint16_t *dst = (uint16_t *)J.dst;
        const float rxf = (float)J.rx, ryf = (float)J.ry, rzf = (float)J.rz;
        if (J.type == 0) {
            const int ic = (int)(l % J.im) + 1;
            const long long r = l / J.im;
            const int jc = (int)(r % J.jm) + 1;
            const int kc = (int)(r / J.jm) + 1;
            const float t1 = ((float)ic - 0.5f) * rxf + 1.0f;
            const float t2 = ((float)jc - 0.5f) * ryf + 1.0f;
            const float t3 = ((float)kc - 0.5f) * rzf + 1.0f;
            dst[cell_index(ic, jc, kc, J.im, J.jm)] =
                (uint16_t)table_coord((R)tex_sample(T, nx, ny, nz, t1, t2, t3), T0, inv_dT, nT);
        } else {
            const int w = J.type - 1;
            float x, y, z;
            if (w <= RC_EAST) {
                const int jc = (int)(l % J.jm) + 1, kc = (int)(l / J.jm) + 1;
                y = ((float)jc - 0.5f) * ryf + 1.0f;
                z = ((float)kc - 0.5f) * rzf + 1.0f;
                x = (w == RC_WEST) ? (J.face ? 1.0f : 1.5f) : (J.face ? (float)imax + 1.0f : (float)imax + 0.5f);
            } else if (w <= RC_NORTH) {
                const int ic = (int)(l % J.im) + 1, kc = (int)(l / J.im) + 1;
                x = ((float)ic - 0.5f) * rxf + 1.0f;
                z = ((float)kc - 0.5f) * rzf + 1.0f;
                y = (w == RC_SOUTH) ? (J.face ? 1.0f : 1.5f) : (J.face ? (float)jmax + 1.0f : (float)jmax + 0.5f);
            } else {
                const int ic = (int)(l % J.im) + 1, jc = (int)(l / J.im) + 1;
                x = ((float)ic - 0.5f) * rxf + 1.0f;
                y = ((float)jc - 0.5f) * ryf + 1.0f;
                z = (w == RC_BOT) ? (J.face ? 1.0f : 1.5f) : (J.face ? (float)kmax + 1.0f : (float)kmax + 0.5f);
            }
            dst[l] = (uint16_t)table_coord((R)tex_sample(T, nx, ny, nz, x, y, z), T0, inv_dT, nT);
        }
    }
}

// ---------------------------------------------------------------------------
// bundle traces: one thread per requested bundle, same device functions
// ---------------------------------------------------------------------------
template <typename R, bool SCAT>
__global__ void k_trace(const DSolve<R> *Sp, int n, const rc_bundle_id *ids, rc_trace_rec *out, int max_cells,
                        int *cells) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    // the descriptor of a finished solve, its run-time fields patched by
    // k_patch_desc before the march
    const DSolve<R> &S = *Sp;
    const rc_bundle_id id = ids[t];
    rc_trace_rec rec;
    rec.nb = rec.g = -1;
    rec.nsteps = 0;
    rec.end_level = 0;
    rec.sx = rec.sy = rec.sz = 0.f;
    rec.tra = 0.f;
    rec.De = 0.0;
    Emitted<R> e;
    const bool ok = emit_bundle(e, S, id.kind, id.i, id.j, id.k, id.v, id.h);
    rec.nb = e.nbg & 0xfffff;
    rec.g = e.nbg >> 20;
    rec.sx = (float)e.sx;
    rec.sy = (float)e.sy;
    rec.sz = (float)e.sz;
    if (ok) {
        Ray<R> r;
        ScatState<R> qs;
        uint4 ctr = make_uint4(0u, 0u, 0u, 0u);
        R ks = (R)0;
        place_bundle(r, S, e);
        if (SCAT) {
            ctr = scatter_counter(S.imax, S.jmax, id.kind, id.i, id.j, id.k, id.v, id.h, 0u);
            ks = scatter_coef(S, e.nbg & 0xfffff, e.nbg >> 20);
            qs.dist = scatter_first_dist(ks > (R)0 ? scatter_first_lnu(S, ctr) : (R)0, ks);
        }
        bool active = level_advance(r, S);
        int ns = 0;
        while (active) {
            if (ns < max_cells && cells) {
                int *c = cells + ((size_t)t * max_cells + ns) * 4;
                c[0] = r.lev;
                c[1] = r.ic;
                c[2] = r.jc;
                c[3] = r.kc;
            }
            march_step<R, SCAT>(r, qs, S);
            if (SCAT && qs.dist < (R)0) scatter_turn(r, ctr, ks, qs, S);
            ns++;
            active = r.tra > r.tol;
            if (active) active = level_advance(r, S);
        }
        rec.nsteps = ns;
        rec.end_level = r.lev;
        rec.tra = (float)r.tra;
        rec.De = r.De;
    }
    out[t] = rec;
}

// Band and g point that emission selects for caller-given uniforms (the
// edge rules of the CDF searches, checked against the oracle and the
// reference's bisection): the same select_band_g the march's emission uses.
template <typename R>
__global__ void k_sample_bands(const DSolve<R> *Sp, int kind, int n, const float *u_b, const float *u_g, int *nb,
                               int *g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int b, q;
    select_band_g(*Sp, kind, (R)u_b[t], (R)u_g[t], b, q);
    nb[t] = b;
    g[t] = q;
}

}  // namespace rc
