// rc_march.cuh -- the persistent march kernel (kernel_fluid + march_ray +
// kernel_surface of src/montecarlo/mc_gpu_noint.cu, restructured for SIMT).
#pragma once
#include "rc_device.cuh"

namespace rc {

// ---------------------------------------------------------------------------
// march: persistent warps over tiles of 32 work items
// ---------------------------------------------------------------------------
//
// A work item is one chunk of rays_per_thread consecutive bundles of one
// (cell, replicate).  A warp takes tiles of 32 items, i.e. pools of
// 32*rays_per_thread bundles:
//   * bundles are emitted in converged waves of 32 (all lanes decode their
//     item and run the Philox draws, direction, band/g search and OERM
//     weights together) into a per-warp ring in shared memory whenever the
//     ring holds fewer than 32 bundles;
//   * every lane traces one ray; the warp steps all its rays until at least
//     kFeedIdle lanes are idle, then hands those lanes the next emitted
//     bundles (warp ballot + prefix count);
//   * two tiles can be in flight: once every bundle of a tile has been
//     emitted, the warp fetches the next tile (of the same solve) and keeps
//     emitting from it while the last rays of the previous tile finish, so
//     long rays do not leave the other lanes idle at tile ends;
//   * each bundle's FP64 tally goes to its own shared-memory slot; when a
//     tile's last bundle has finished, its slots are summed in bundle
//     order, so the result does not depend on which lane traced which
//     bundle.
// Shared memory per warp is the ring (64 emitted bundles of 32 bytes: the
// start position is rebuilt from the emitting cell when a lane takes the
// bundle) and two slot arrays; everything else stays in L1-cached global
// memory, so that most of the SM's 256 KB of L1/shared storage caches the
// temperature pyramid and the k / I_b tables (48-byte entries, an earlier
// layout, were 1.2% slower; 64-byte entries 4%).  The scattering variant
// keeps these entries and adds a small side array (see WarpShared).

struct MarchArgs {
    const void *solves;          // DSolve<R>[nsolves] (run-time fields patched on the device)
    const long long *tile_start; // [nsolves+1] exclusive prefix of tiles
    int nsolves;
    long long total_tiles;
    unsigned long long *tile_counter;
    int rpt_max;
    // long-ray priority (one solve only; NULL: tiles in natural order): the
    // first *n_prio claims take prio_tiles[], the rest take the natural
    // order and skip the tiles whose tile_prio byte is set
    const unsigned *prio_tiles;
    const unsigned char *tile_prio;
    const unsigned *n_prio;
};

// Long-ray priority list.  A bundle whose path is long -- nearly parallel
// to the x walls, so that it runs between the periodic y/z boundaries, and
// in a near-transparent band, so that its transmissivity stays above the
// cutoff -- takes up to the last level's step budget; a launch that starts
// it late idles while it finishes.  The march therefore claims the tiles
// holding such a bundle first.  The estimate of a bundle's path length is
//   L = min(d_x / |s_x|, ln(1/tol) / k_min),
// d_x the distance from its start to the x wall it moves towards, k_min the
// smallest absorption coefficient of its band and g point over the table
// rows the field's temperatures span (k_prio_kmin); a tile is listed when
// some bundle has L > thr * Lx.  The draws are the emission's own (Philox
// counter of the bundle, select_band_g), so the estimate sees the same
// direction, band and g point the march will trace.  Only the order in
// which tiles are claimed changes, never a result.
template <typename R>
__global__ void k_prio_kmin(const DSolve<R> *Sp, float *kmin) {
    const DSolve<R> &S = *Sp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.nB * S.nQ) return;
    const double T0 = S.sc->T0, idt = S.sc->inv_dT;
    const double tmin = (double)__uint_as_float(S.sc->tmin_bits), tmax = (double)__uint_as_float(S.sc->tmax_bits);
    const int lo = max(0, min(S.nT - 1, (int)floor((tmin - T0) * idt)));
    const int hi = max(lo, min(S.nT - 1, (int)floor((tmax - T0) * idt) + 1));
    float k = 3.0e38f;
    for (int t = lo; t <= hi; ++t) k = fminf(k, (float)S.ki[(size_t)i * S.nT + t].k0);
    kmin[i] = fmaxf(k, 0.f);
}

template <typename R>
__global__ void k_prio_tiles(const DSolve<R> *Sp, float thr, const float *kmin, unsigned *prio_tiles,
                             unsigned char *tile_prio, unsigned *n_prio) {
    const DSolve<R> &S = *Sp;
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    const float Lx = (float)S.Lx, Lthr = thr * Lx;
    const float tau_f = logf(1.0f / fmaxf((float)S.toll, 1e-30f)), tau_w = logf(1.0f / fmaxf((float)S.tollS, 1e-30f));
    for (long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile < S.n_tiles;
         tile += nw) {
        const ItemId it = decode_item(S, tile * kWarp + lane);
        bool cand = false;
        if (it.kind >= 0) {
            const uint32_t cell = (it.kind == 0)
                                      ? (uint32_t)((it.i - 1) + S.imax * ((it.j - 1) + S.jmax * (it.k - 1)))
                                      : (uint32_t)((it.j - 1) + S.jmax * (it.k - 1));
            const float x0 = it.kind == 0 ? (float)S.xc[it.i] : (it.kind == 1 ? 0.f : Lx);
            const float tau = it.kind == 0 ? tau_f : tau_w;
            const int h1 = min(it.h0 + S.rpt, S.photmax);
            for (int h = it.h0; h < h1 && !cand; ++h) {
                const rc_u32x4 d = bundle_draws(S.key0, S.key1, h, it.v, it.kind, cell);
                const float u = rc_u01(d.y);
                // s_x as emit_bundle draws it: 1 - 2u (fluid), sqrt(1 - u) / -sqrt(u) (walls)
                const float sx = it.kind == 0 ? 1.f - 2.f * u : (it.kind == 1 ? sqrtf(1.f - u) : -sqrtf(u));
                const float dx = sx > 0.f ? Lx - x0 : x0;
                const float Lw = dx / fmaxf(fabsf(sx), 1e-10f);
                if (!(Lw > Lthr)) continue;
                int nb, g;
                select_band_g(S, it.kind, (R)rc_u01(d.z), (R)rc_u01(d.w), nb, g);
                const float k = kmin[nb * S.nQ + g];
                cand = k * Lthr < tau;  // ln(1/tol) / k > Lthr
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, cand);
        if (lane == 0) {
            tile_prio[tile] = m != 0u;
            if (m) prio_tiles[atomicAdd(n_prio, 1u)] = (unsigned)tile;
        }
    }
}

template <typename R, bool SCAT>
struct WarpShared {
    Emitted<R> ring[kRing];
};
// With scattering, also the free path to the first event of every ring
// entry (drawn by the emission wave), and the scattering coefficient and
// event count of every lane's bundle (read and written by that lane only,
// at placement and at events; its counter words are decoded again from its
// work item at an event).  The ring entries keep their 32 bytes.
template <typename R>
struct WarpShared<R, true> {
    Emitted<R> ring[kRing];
    R dist[kRing];
    R ks[kWarp];
    uint32_t nev[kWarp];
};

// Index of the solve owning a global tile (tile_start is an exclusive prefix).
__device__ __forceinline__ int solve_of_tile(const long long *tile_start, int nsolves, unsigned long long tile) {
    int lo = 0, hi = nsolves;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned long long)tile_start[mid] <= tile) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void flush_counters(DScalars *sc, unsigned long long &nsteps, unsigned long long &nbund,
                                               int lane) {
    unsigned long long st = nsteps, nb = nbund;
    for (int o = 16; o > 0; o >>= 1) {
        st += __shfl_xor_sync(0xffffffffu, st, o);
        nb += __shfl_xor_sync(0xffffffffu, nb, o);
    }
    if (lane == 0) {
        atomicAdd(&sc->steps, st);
        atomicAdd(&sc->bundles, nb);
    }
    nsteps = nbund = 0;
}

// MINB: resident 256-thread blocks per SM the register allocation must
// allow (2: up to 128 registers, 3: 80, 4: 64).  SCAT: the variant for
// media with scattering particles (solves without them run in it unchanged).
template <typename R, int MINB, bool SCAT>
__global__ void __launch_bounds__(256, MINB) k_march(MarchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    WarpShared<R, SCAT> *ws = reinterpret_cast<WarpShared<R, SCAT> *>(smem) + warp;
    const size_t wbytes = ((sizeof(WarpShared<R, SCAT>) * nwarps) + 15) & ~(size_t)15;
    const int pool_max = kWarp * a.rpt_max;
    double *slots0 = reinterpret_cast<double *>(smem + wbytes) + (size_t)warp * 2 * pool_max;
    const DSolve<R> *solves = reinterpret_cast<const DSolve<R> *>(a.solves);
    const unsigned lt = (1u << lane) - 1u;
    const DSolve<R> *Sp = solves;

    // warp-uniform state
    int cur_solve = -1;
    long long item0_0 = 0, item0_1 = 0;  // first item of the tile in each buffer
    unsigned busy = 0u;     // bit p: buffer p holds a tile not yet reduced
    unsigned emitted = 0u;  // bit p: every bundle of buffer p's tile emitted
    int out0 = 0, out1 = 0; // emitted bundles of each buffer not finished yet
    int epar = -1;          // buffer being emitted from
    int next_b = 0, head = 0, count = 0;
    bool drained = false;   // no more tiles
    unsigned long long pending = ~0ull;  // fetched tile waiting for a solve switch
    // tiles claimed from the queue but not started: [chunk_next, chunk_end)
    unsigned long long chunk_next = 0, chunk_end = 0;
    // with the long-ray priority list, the claim space is the listed tiles
    // followed by all tiles in natural order (listed ones skipped there)
    const unsigned long long nprio = a.n_prio ? (unsigned long long)__ldg(a.n_prio) : 0ull;
    const unsigned long long total = (unsigned long long)a.total_tiles + nprio;
    const unsigned long long all_warps = (unsigned long long)gridDim.x * nwarps;
    // lanes tracing a ray, and lanes whose ray belongs to buffer 1
    // (warp-uniform; kept in step with the lanes' own flags)
    unsigned amask = 0u, p1mask = 0u;
    // lane state
    bool active = false;
    int myslot = 0;  // slot of the lane's bundle: parity * pool_max + index
    unsigned long long nsteps = 0, nbund = 0;
    Ray<R> r;
    ScatState<R> qs;

    for (;;) {
        // ---- fetch the next tile into a free buffer
        if (!drained && (epar < 0 || ((emitted >> epar) & 1u))) {
            const int fpar = (epar < 0) ? 0 : (epar ^ 1);
            if (!((busy >> fpar) & 1u)) {
                unsigned long long tile = pending;
                if (tile == ~0ull) {
                    // ends: every pass advances chunk_next or the shared
                    // counter, and a claim at or past `total` ends the queue
                    for (;;) {
                        if (chunk_next >= chunk_end) {
                            // guided self-scheduling: claim up to kChunkMax
                            // consecutive tiles (usually of one solve), so a
                            // warp keeps two tiles of the same solve in
                            // flight; claim fewer as the queue drains to keep
                            // the tail short
                            unsigned long long c0 = 0;
                            if (lane == 0) {
                                const unsigned long long seen = *(volatile unsigned long long *)a.tile_counter;
                                const unsigned long long rem = seen < total ? total - seen : 0ull;
                                const unsigned long long k =
                                    max(1ull, min((unsigned long long)kChunkMax, rem / (4ull * all_warps)));
                                c0 = atomicAdd(a.tile_counter, k);
                                chunk_end = min(c0 + k, total);
                            }
                            c0 = __shfl_sync(0xffffffffu, c0, 0);
                            chunk_end = __shfl_sync(0xffffffffu, chunk_end, 0);
                            chunk_next = c0;
                        }
                        tile = chunk_next < chunk_end ? chunk_next++ : total;
                        if (!a.n_prio || tile >= total) break;
                        if (tile < nprio) {
                            tile = __ldg(a.prio_tiles + tile);
                            break;
                        }
                        if (!__ldg(a.tile_prio + (tile - nprio))) {
                            tile -= nprio;
                            break;
                        }
                        // a listed tile met again in natural order: claim the next
                    }
                }
                if (tile >= (unsigned long long)a.total_tiles) {
                    drained = true;
                    pending = ~0ull;
                } else {
                    const int so = solve_of_tile(a.tile_start, a.nsolves, tile);
                    if (so != cur_solve && busy) {
                        pending = tile;  // switch solves only once both buffers are reduced
                    } else {
                        pending = ~0ull;
                        if (so != cur_solve) {
                            if (cur_solve >= 0) flush_counters(Sp->sc, nsteps, nbund, lane);
                            Sp = solves + so;
                            cur_solve = so;
                        }
                        const long long i0 =
                            ((long long)(tile - (unsigned long long)a.tile_start[so]) + Sp->tile_base) * kWarp;
                        if (fpar) item0_1 = i0;
                        else item0_0 = i0;
                        double *sl = slots0 + fpar * pool_max;
                        for (int b = lane; b < kWarp * Sp->rpt; b += kWarp) sl[b] = 0.0;
                        busy |= 1u << fpar;
                        emitted &= ~(1u << fpar);
                        if (fpar) out1 = 0;
                        else out0 = 0;
                        epar = fpar;
                        next_b = 0;
                        __syncwarp();
                    }
                }
            }
        }
        const DSolve<R> &S = *Sp;
        const int rpt = S.rpt;
        const int lrpt = __ffs(rpt) - 1;  // rpt is a power of two
        const int pool = kWarp * rpt;
        // ---- converged emission wave: one bundle per lane
        if (count < kWarp && epar >= 0 && !((emitted >> epar) & 1u)) {
            const int b = next_b + lane;
            Emitted<R> e;
            R dist0 = (R)kNoEvent;
            bool ok = false;
            if (b < pool) {
                const ItemId it = decode_item(S, (epar ? item0_1 : item0_0) + (b >> lrpt));
                const int h = it.h0 + (b & (rpt - 1));
                if (it.kind >= 0 && h < S.photmax) {
                    nbund++;
                    // with particles, draw 1 (scatter_first_lnu, written
                    // out: the call form spilled) before the emission
                    // itself: little is live then, so the variant fits the
                    // register budget without spilling
                    R lnu = (R)0;
                    if constexpr (SCAT) {
                        if (S.nA > 0) {
                            const uint4 c0 = scatter_counter(S.imax, S.jmax, it.kind, it.i, it.j, it.k, it.v, h, 0u);
                            rc_u32x4 c;
                            c.x = c0.x;
                            c.y = c0.y;
                            c.z = c0.z;
                            c.w = 1u;
                            const rc_u32x4 d = rc_philox4x32_10(c, S.key0, S.key1);
                            lnu = -RT<R>::log_((R)rc_u01(d.x));
                        }
                    }
                    ok = emit_bundle(e, S, it.kind, it.i, it.j, it.k, it.v, h);
                    e.kk |= (b << 18) | (epar << 29);
                    if constexpr (SCAT) {
                        const R ks = scatter_coef(S, e.nbg & 0xfffff, e.nbg >> 20);
                        if (ks > (R)0) dist0 = lnu / ks;  // scatter_first_dist
                    }
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            int pos = __popc(m & lt);
            if (S.sort) {
                // band-sorted order: the wave enters the ring by ascending
                // k_{nb,g} at the table row nearest Tmax (ties by lane), so
                // bundles handed out together have similar optical path
                // lengths.  Which lane traces a bundle does not change its
                // tally (each bundle owns its slot).
                unsigned key = 0xffffffffu;
                if (ok) {
                    const int nb = e.nbg & 0xfffff, g = e.nbg >> 20;
                    key = __float_as_uint((float)S.ki[RC_IX(((size_t)nb * S.nQ + g) * S.nT + S.row,
                                                            (long long)S.nB * S.nQ * S.nT, SITE_EMIT_ROW, S)]
                                              .k0);  // k >= 0: monotone bits
                }
                int rank = 0;
                for (int q = 0; q < kWarp; ++q) {
                    const unsigned kq = __shfl_sync(0xffffffffu, key, q);
                    rank += (kq < key) || (kq == key && q < lane);
                }
                pos = rank;
            }
            if (ok) {
                ws->ring[(head + count + pos) & (kRing - 1)] = e;
                if constexpr (SCAT) ws->dist[(head + count + pos) & (kRing - 1)] = dist0;
            }
            count += __popc(m);
            if (epar) out1 += __popc(m);
            else out0 += __popc(m);
            next_b += kWarp;
            if (next_b >= pool) emitted |= 1u << epar;
            __syncwarp();
        }
        // ---- idle lanes take emitted bundles
        {
            const unsigned m = ~amask;
            const int navail = min(count, __popc(m));
            bool took = false, fin = false;
            if (!active) {
                const int rank = __popc(m & lt);
                if (rank < navail) {
                    const Emitted<R> &e = ws->ring[(head + rank) & (kRing - 1)];
                    place_bundle(r, S, e);
                    if constexpr (SCAT) {
                        qs.dist = ws->dist[(head + rank) & (kRing - 1)];
                        ws->ks[lane] = scatter_coef(S, e.nbg & 0xfffff, e.nbg >> 20);
                        ws->nev[lane] = 0u;
                    }
                    myslot = ((e.kk >> 29) & 1) * pool_max + ((e.kk >> 18) & 0x7ff);
                    took = true;
                    active = level_advance(r, S);
                    if (!active) {
                        slots0[myslot] = r.De;
                        fin = true;
                    }
                }
            }
            head = (head + navail) & (kRing - 1);
            count -= navail;
            if (navail > 0) {
                const unsigned tk = __ballot_sync(0xffffffffu, took);
                const unsigned t1 = __ballot_sync(0xffffffffu, took && myslot >= pool_max);
                const unsigned fi = __ballot_sync(0xffffffffu, fin);
                p1mask = (p1mask & ~tk) | t1;
                amask = (amask | tk) & ~fi;
                out1 -= __popc(fi & t1);
                out0 -= __popc(fi & ~t1);
            }
            __syncwarp();
        }
        // ---- step every active ray; stay in this loop until enough lanes
        //      are idle to be worth handing out bundles (or a tile can be
        //      reduced, or every lane is idle)
        {
            const bool can_feed =
                count > 0 || (epar >= 0 && !((emitted >> epar) & 1u)) ||
                (!drained && (epar < 0 || (((emitted >> epar) & 1u) && !((busy >> (epar ^ 1)) & 1u))));
            for (;;) {
                bool fin = false;
                bool wait_turn = false;
                if constexpr (SCAT) wait_turn = active && qs.dist < (R)0;
                if (active && !wait_turn) {
                    const int budget = march_step<R, SCAT>(r, qs, S);
                    nsteps++;
                    bool done = !(r.tra > r.tol);
                    if (!done && r.counter >= budget) done = !level_advance(r, S);
                    if (done) {
                        slots0[myslot] = r.De;
                        active = false;
                        fin = true;
                    }
                    if constexpr (SCAT) wait_turn = active && qs.dist < (R)0;
                }
                const unsigned fm = __ballot_sync(0xffffffffu, fin);
                if (fm) {
                    const int n1 = __popc(fm & p1mask);
                    out1 -= n1;
                    out0 -= __popc(fm) - n1;
                    amask &= ~fm;
                }
                // lanes stopped at a scattering event wait for a turn pass,
                // which draws all their new directions at once; the pass is
                // long and runs on the waiting lanes only, so it waits until
                // kTurnGather lanes wait, or every traced ray does
                unsigned tm = 0u;
                bool turn_now = false;
                if constexpr (SCAT) {
                    tm = __ballot_sync(0xffffffffu, wait_turn);
                    turn_now = __popc(tm) >= kTurnGather || (tm && !(amask & ~tm));
                }
                const int nidle = kWarp - __popc(amask & ~tm);
                if (nidle == kWarp) break;
                if (nidle >= kFeedIdle && (can_feed || turn_now)) break;
                if (fm && ((((busy & emitted) & 1u) && out0 == 0) || (((busy & emitted) & 2u) && out1 == 0))) break;
            }
        }
        // ---- scattering: the new directions of every lane stopped at an
        //      event, once kTurnGather lanes wait or no traced ray is left
        //      that does not wait (waiting lanes never deadlock the warp)
        if constexpr (SCAT) {
            const unsigned tw = __ballot_sync(0xffffffffu, active && qs.dist < (R)0);
            const bool turn_now = __popc(tw) >= kTurnGather || (tw && !(amask & ~tw));
            if (turn_now && active && qs.dist < (R)0) {
                const int mypar = myslot >= pool_max, myb = myslot - mypar * pool_max;
                const ItemId it = decode_item(S, (mypar ? item0_1 : item0_0) + (myb >> lrpt));
                uint4 c = scatter_counter(S.imax, S.jmax, it.kind, it.i, it.j, it.k, it.v, it.h0 + (myb & (rpt - 1)),
                                          ws->nev[lane]);
                scatter_turn(r, c, ws->ks[lane], qs, S);
                ws->nev[lane] = c.w;
            }
        }
        // ---- reduce finished tiles: chunk sums in bundle order, group sums
        //      in item order
#pragma unroll
        for (int par = 0; par < 2; ++par) {
            const int outp = par ? out1 : out0;
            if (((busy & emitted) >> par) & 1u && outp == 0) {
                __syncwarp();
                const double *sl = slots0 + par * pool_max;
                double s = 0.0;
                for (int h = 0; h < rpt; ++h) s += sl[lane * rpt + h];
                const int gs = S.gsize;
                const int base = (lane / gs) * gs;
                double g = 0.0;
                for (int q = 0; q < gs; ++q) g += __shfl_sync(0xffffffffu, s, base + q);
                const long long item = (par ? item0_1 : item0_0) + lane;
                if (lane == base && item < S.n_items) S.partial[RC_IX(item / gs, S.n_partial, SITE_PARTIAL, S)] = g;
                busy &= ~(1u << par);
                if (epar == par) epar = -1;
                __syncwarp();
            }
        }
        if (drained && !busy) break;
    }
    if (cur_solve >= 0) flush_counters(Sp->sc, nsteps, nbund, lane);
}

template <typename R, bool SCAT>
constexpr size_t march_smem_bytes(int block, int rpt_max) {
    return ((((size_t)sizeof(WarpShared<R, SCAT>) * (block / kWarp)) + 15) & ~(size_t)15) +
           (size_t)(block / kWarp) * 2 * kWarp * rpt_max * sizeof(double);
}

}  // namespace rc
