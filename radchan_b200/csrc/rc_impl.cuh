// rc_impl.cuh -- solver contexts and the per-solve pipeline on one stream,
// shared by rc_solver.cu (C ABI, batches, traces, autotuner) and
// rc_server.cu (continuous-batching server).
//
// Replaces the host side of the reference (mc_gpu_, get_results_,
// memory_copy_noint.cu): the grid, the tables and the Planck table are
// uploaded once per context and stay resident; a solve copies only the
// temperature field and runs
//   k_init_scalars -> k_tmax -> k_setup1 -> [k_grey_ib] -> k_setup2 ->
//   k_levels -> k_patch_desc -> k_march -> k_tally_multi
// on the context's stream without any host synchronisation.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "rc_host.h"
#include "rc_kernels.cuh"

#pragma once

using namespace rc;

namespace rc_detail {

// Host-side failure injection (rc_debug_fail_next): a named site reached
// while armed fails as if its CUDA call had returned an error, without
// making the call, so error paths and recovery are tested with no device
// fault.  Sites: field_copy, march, tally, collect, dns, quantum.
struct FailPoints {
    std::atomic<int> armed{0};
    std::mutex mu;
    std::map<std::string, int> left;
};
inline FailPoints &fail_points() {
    static FailPoints f;
    return f;
}
inline bool fail_now(const char *site) {
    FailPoints &f = fail_points();
    if (!f.armed.load(std::memory_order_relaxed)) return false;
    std::lock_guard<std::mutex> lk(f.mu);
    auto it = f.left.find(site);
    if (it == f.left.end() || it->second <= 0) return false;
    if (--it->second == 0) {
        f.left.erase(it);
        f.armed.fetch_sub(1);
    }
    return true;
}

// NVTX range over a host scope (solve enqueue, collect, batch, server
// quantum, DNS coupling): a profiler shows the kernels each one launched
// under its name; without a profiler attached the calls do nothing.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};
}  // namespace rc_detail

#define RC_CK(call)                                                                                    \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return set_err(err_, RC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

#define RC_FAILPOINT(site)                                                                             \
    do {                                                                                               \
        if (fail_now(site)) return set_err(err_, RC_E_CUDA, std::string("injected failure at ") + site); \
    } while (0)

// ---------------------------------------------------------------------------
// context implementation, templated on the march precision
// ---------------------------------------------------------------------------
namespace rc_detail {
struct TallyOut {
    double *q64, *var64, *qw64, *vw64;
    float *Qc, *Sc, *Wq, *Ws;
};

// Replicate sums -> per-cell mean and variance of the mean
// (kernel_fluid :229-239, kernel_surface :1468-1478), into compact FP64 and
// FP32 outputs; one solve per blockIdx.y.
template <typename R>
__global__ void k_tally_multi(const DSolve<R> *solves, const TallyOut *outs) {
    const int s = blockIdx.y;
    const TallyOut &o = outs[s];
    const DSolve<R> &S = solves[s];
    const long long ncf = (long long)S.imax * S.jmax * S.kloc;
    const long long ncw = (long long)S.nwalls * S.jmax * S.kloc;
    const int nVar = S.nVar, np = S.nparts;
    double a = 0.0;
    if (nVar > 1) {
        a = 1. / (nVar - 0.5);
        a = a * 1. / (nVar - 1);
    }
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncf + ncw;
         c += (long long)gridDim.x * blockDim.x) {
        const double *p = S.partial + c * nVar * np;
        double sum = 0.0;
        for (int v = 0; v < nVar; ++v) {
            double dv = 0.0;
            for (int q = 0; q < np; ++q) dv += p[v * np + q];
            sum += dv;
        }
        const double mean = sum / nVar;
        double var = 0.0;
        for (int v = 0; v < nVar; ++v) {
            double dv = 0.0;
            for (int q = 0; q < np; ++q) dv += p[v * np + q];
            const double d = dv - mean;
            var += a * d * d;
        }
        if (c < ncf) {
            if (o.q64) o.q64[c] = mean;
            if (o.var64) o.var64[c] = var;
            o.Qc[c] = (float)mean;
            o.Sc[c] = (float)sqrt(var);
        } else {
            const long long cw = c - ncf;
            const long long nwc = (long long)S.jmax * S.kloc;
            const int slot = (int)(cw / nwc);
            const long long off = (long long)S.wall_id[slot] * nwc + (cw % nwc);
            if (o.qw64) o.qw64[off] = mean;
            if (o.vw64) o.vw64[off] = var;
            o.Wq[off] = (float)mean;
            o.Ws[off] = (float)sqrt(var);
        }
    }
}

struct ImplBase {
    virtual ~ImplBase() {}
};

// Many copies in one launch: segment blockIdx.y copies n floats from src to
// dst (a batch's fields from the members' pinned staging, which the device
// reads directly, and its results into one buffer for one copy to the host).
struct CopySeg {
    const float *src;
    float *dst;
    long long n;
};
static __global__ void k_copy_segs(const CopySeg *segs) {
    const CopySeg s = segs[blockIdx.y];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < s.n; i += (long long)gridDim.x * blockDim.x)
        s.dst[i] = s.src[i];
}

struct SlotCommon {
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e_march0 = nullptr, e_march1 = nullptr;
    cudaEvent_t e_dns = nullptr;  // end of a DNS-source kernel on another stream
    float *d_T = nullptr, *h_T = nullptr;
    DScalars *d_sc = nullptr, *h_sc = nullptr;
    double *d_partial = nullptr;
    size_t partial_cap = 0;
    double *d_q64 = nullptr, *d_var64 = nullptr, *d_qw64 = nullptr, *d_vw64 = nullptr;
    float *d_Qc = nullptr, *d_Sc = nullptr, *d_Wq = nullptr, *d_Ws = nullptr;
    float *h_Qc = nullptr, *h_Sc = nullptr, *h_Wq = nullptr, *h_Ws = nullptr;
    long long *d_tiles = nullptr, *h_tiles = nullptr;
    unsigned long long *d_counter = nullptr;
    TallyOut *d_out = nullptr, *h_out = nullptr;
    // long-ray priority list (k_prio_tiles): listed tiles, per-tile flag,
    // count, and the smallest k of every band and g point over the field's
    // temperature range (k_prio_kmin)
    unsigned *d_prio = nullptr, *d_nprio = nullptr;
    unsigned char *d_tprio = nullptr;
    float *d_kmin = nullptr;
    long long prio_cap = 0;
    int kmin_cap = 0;
    // what the list was built for: the work decomposition and the draws; the
    // list is kept while those stay the same (a later field only changes how
    // well it orders the work, never a result)
    long long prio_key[10] = {};
    bool prio_ok = false;
    int state = 0;  // 0 free, 1 in flight, 2 finished (results pending)
    rc_ticket ticket = -1;
    int zstart = 1;
    int rpt = 0, block = 0;
    bool host_copied = false;
};

}  // namespace rc_detail

struct rc_ctx {
    rc_params p;
    int device = 0;
    int wt[6];
    int kloc = 0;
    std::vector<GridLevel> grid;
    std::string err;
    int next_ticket = 1;
    // launch knobs
    int rpt = 8, block = 256, sort = 0, minb = 3;
    float prio_thr = RC_PRIORITY_DEFAULT;  // long-ray priority: estimated path length in units of Lx (0: off)
    int num_sms = 148;
    bool has_tables = false;
    // changes with every call that changes what a solve's descriptor holds
    // (tables, particles, launch knobs): a batch captured before such a
    // change is captured again
    unsigned long long gen = 0;
    // DNS-coupling scratch (rc_dns_source): T1 pencil + four outputs, and a counter
    double *d_dns = nullptr;
    size_t dns_cap = 0;
    unsigned long long *d_dns_n = nullptr;
    double *h_dns = nullptr;  // pinned staging of the same arrays
    size_t dns_hcap = 0;
    // precision-specific state
    void *impl = nullptr;  // Impl<float> or Impl<double>
    int dbl = 0;
};

namespace rc_detail {

template <typename R>
struct Slot : SlotCommon {
    uint16_t *d_levAll = nullptr;      // every level's table coordinates (one allocation)
    std::vector<uint16_t *> d_levT;    // per-level views into d_levAll
    uint16_t *d_lw[RC_MAX_LEVELS][6] = {};
    uint16_t *d_Tw0[2] = {nullptr, nullptr};
    KIRow<R> *d_ki_grey = nullptr;
    R *d_cdf_f = nullptr, *d_cdf_s = nullptr, *d_den_f = nullptr, *d_ibm = nullptr;
    int *d_guide_f = nullptr, *d_guide_s = nullptr;
    R *d_Tnb_grey = nullptr, *d_Ibt_grey = nullptr;
    DSolve<R> *d_desc = nullptr, *h_desc = nullptr;
    LevelJobs jobs;
};

template <typename R>
struct Impl : ImplBase {
    rc_ctx *c = nullptr;
    R *d_faces = nullptr;              // every level's xu | yu | zu (one allocation)
    std::vector<R *> d_xu, d_yu, d_zu; // per-level views into d_faces
    std::vector<int> face_off, lev_off;  // per-level offsets in d_faces / Slot::d_levAll
    long long n_faces = 0, n_pyramid = 0;  // their lengths
    R *d_xc = nullptr, *d_yc = nullptr, *d_zc = nullptr;
    R *d_kt = nullptr, *d_Ibt = nullptr, *d_probg = nullptr, *d_prob = nullptr, *d_probq = nullptr;
    R *d_Ibw = nullptr, *d_Tnb = nullptr, *d_kP = nullptr, *d_wvl = nullptr, *d_wvr = nullptr, *d_wvc = nullptr;
    KIRow<R> *d_ki = nullptr;
    int nT = 0, nB = 0, nQ = 0;
    // scattering particles (rc_set_scattering): coefficient, phase CDF, angles in turns
    R *d_ksca = nullptr, *d_pcdf = nullptr, *d_pth = nullptr;
    uint16_t *d_pguide = nullptr;
    int nA = 0;
    std::vector<Slot<R>> slots;
    int smem_opt_in = 0;

    ~Impl() override { release(); }

    template <typename T>
    static void dfree(T *&p) {
        if (p) cudaFree((void *)p);
        p = nullptr;
    }
    template <typename T>
    static void hfree(T *&p) {
        if (p) cudaFreeHost((void *)p);
        p = nullptr;
    }

    void release_tables() {
        dfree(d_kt);
        dfree(d_Ibt);
        dfree(d_probg);
        dfree(d_prob);
        dfree(d_probq);
        dfree(d_Ibw);
        dfree(d_Tnb);
        dfree(d_kP);
        dfree(d_wvl);
        dfree(d_wvr);
        dfree(d_wvc);
        dfree(d_ki);
        release_scattering();
    }

    void release_scattering() {
        dfree(d_ksca);
        dfree(d_pcdf);
        dfree(d_pth);
        dfree(d_pguide);
        nA = 0;
    }

    void release() {
        for (auto &s : slots) {
            if (s.st) cudaStreamSynchronize(s.st);
            dfree(s.d_T);
            hfree(s.h_T);
            dfree(s.d_sc);
            hfree(s.h_sc);
            dfree(s.d_partial);
            dfree(s.d_q64);
            dfree(s.d_var64);
            dfree(s.d_qw64);
            dfree(s.d_vw64);
            dfree(s.d_Qc);
            dfree(s.d_Sc);
            dfree(s.d_Wq);
            dfree(s.d_Ws);
            hfree(s.h_Qc);
            hfree(s.h_Sc);
            hfree(s.h_Wq);
            hfree(s.h_Ws);
            dfree(s.d_tiles);
            hfree(s.h_tiles);
            dfree(s.d_counter);
            dfree(s.d_out);
            hfree(s.h_out);
            dfree(s.d_prio);
            dfree(s.d_tprio);
            dfree(s.d_nprio);
            dfree(s.d_kmin);
            s.prio_cap = 0;
            s.kmin_cap = 0;
            s.prio_ok = false;
            dfree(s.d_levAll);
            s.d_levT.clear();
            for (int l = 0; l < RC_MAX_LEVELS; ++l)
                for (int w = 0; w < 6; ++w) dfree(s.d_lw[l][w]);
            dfree(s.d_Tw0[0]);
            dfree(s.d_Tw0[1]);
            dfree(s.d_ki_grey);
            dfree(s.d_cdf_f);
            dfree(s.d_cdf_s);
            dfree(s.d_den_f);
            dfree(s.d_ibm);
            dfree(s.d_guide_f);
            dfree(s.d_guide_s);
            dfree(s.d_Tnb_grey);
            dfree(s.d_Ibt_grey);
            dfree(s.d_desc);
            hfree(s.h_desc);
            if (s.e0) cudaEventDestroy(s.e0);
            if (s.e1) cudaEventDestroy(s.e1);
            if (s.e_march0) cudaEventDestroy(s.e_march0);
            if (s.e_march1) cudaEventDestroy(s.e_march1);
            if (s.e_dns) cudaEventDestroy(s.e_dns);
            if (s.st) cudaStreamDestroy(s.st);
        }
        slots.clear();
        dfree(d_faces);
        d_xu.clear();
        d_yu.clear();
        d_zu.clear();
        dfree(d_xc);
        dfree(d_yc);
        dfree(d_zc);
        release_tables();
    }

    template <typename T>
    int upload(T *&dst, const std::vector<float> &src, std::string *err_) {
        std::vector<T> tmp(src.begin(), src.end());
        RC_CK(cudaMalloc((void **)&dst, std::max<size_t>(1, tmp.size()) * sizeof(T)));
        if (!tmp.empty()) RC_CK(cudaMemcpy(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
        return RC_OK;
    }

    int init(int nslots) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        const int nl = p.grid_num;
        d_xu.assign(nl, nullptr);
        d_yu.assign(nl, nullptr);
        d_zu.assign(nl, nullptr);
        face_off.assign(nl, 0);
        lev_off.assign(nl, 0);
        {
            std::vector<float> faces;
            long long po = 0;
            for (int l = 0; l < nl; ++l) {
                const GridLevel &g = c->grid[l];
                face_off[l] = (int)faces.size();
                faces.insert(faces.end(), g.xu.begin(), g.xu.end());
                faces.insert(faces.end(), g.yu.begin(), g.yu.end());
                faces.insert(faces.end(), g.zu.begin(), g.zu.end());
                lev_off[l] = (int)po;
                po += (long long)p.maxi[l] * p.maxj[l] * p.maxk[l];
                if (po > 0x7fffffffLL) return set_err(err_, RC_E_INVALID, "grid too large for 32-bit level offsets");
            }
            n_faces = (long long)faces.size();
            n_pyramid = po;
            int rc = upload(d_faces, faces, err_);
            if (rc) return rc;
            for (int l = 0; l < nl; ++l) {
                d_xu[l] = d_faces + face_off[l];
                d_yu[l] = d_xu[l] + (p.maxi[l] + 1);
                d_zu[l] = d_yu[l] + (p.maxj[l] + 1);
            }
        }
        int rc = upload(d_xc, c->grid[0].x, err_);
        if (!rc) rc = upload(d_yc, c->grid[0].y, err_);
        if (!rc) rc = upload(d_zc, c->grid[0].z, err_);
        if (rc) return rc;
        slots.resize(nslots);
        const size_t nfield = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
        const size_t ncf = (size_t)p.imax * p.jmax * c->kloc;
        const size_t nwc = (size_t)2 * p.jmax * c->kloc;
        for (auto &s : slots) {
            RC_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
            RC_CK(cudaEventCreate(&s.e0));
            RC_CK(cudaEventCreate(&s.e1));
            RC_CK(cudaEventCreate(&s.e_march0));
            RC_CK(cudaEventCreate(&s.e_march1));
            RC_CK(cudaMalloc((void **)&s.d_T, nfield * sizeof(float)));
            RC_CK(cudaHostAlloc((void **)&s.h_T, nfield * sizeof(float), cudaHostAllocDefault));
            RC_CK(cudaMalloc((void **)&s.d_sc, sizeof(DScalars)));
            RC_CK(cudaHostAlloc((void **)&s.h_sc, sizeof(DScalars), cudaHostAllocDefault));
            RC_CK(cudaMalloc((void **)&s.d_q64, ncf * sizeof(double)));
            RC_CK(cudaMalloc((void **)&s.d_var64, ncf * sizeof(double)));
            RC_CK(cudaMalloc((void **)&s.d_qw64, nwc * sizeof(double)));
            RC_CK(cudaMalloc((void **)&s.d_vw64, nwc * sizeof(double)));
            RC_CK(cudaMalloc((void **)&s.d_Qc, ncf * sizeof(float)));
            RC_CK(cudaMalloc((void **)&s.d_Sc, ncf * sizeof(float)));
            RC_CK(cudaMalloc((void **)&s.d_Wq, nwc * sizeof(float)));
            RC_CK(cudaMalloc((void **)&s.d_Ws, nwc * sizeof(float)));
            RC_CK(cudaMemset(s.d_Wq, 0, nwc * sizeof(float)));
            RC_CK(cudaMemset(s.d_Ws, 0, nwc * sizeof(float)));
            RC_CK(cudaMemset(s.d_qw64, 0, nwc * sizeof(double)));
            RC_CK(cudaMemset(s.d_vw64, 0, nwc * sizeof(double)));
            RC_CK(cudaHostAlloc((void **)&s.h_Qc, ncf * sizeof(float), cudaHostAllocDefault));
            RC_CK(cudaHostAlloc((void **)&s.h_Sc, ncf * sizeof(float), cudaHostAllocDefault));
            RC_CK(cudaHostAlloc((void **)&s.h_Wq, nwc * sizeof(float), cudaHostAllocDefault));
            RC_CK(cudaHostAlloc((void **)&s.h_Ws, nwc * sizeof(float), cudaHostAllocDefault));
            RC_CK(cudaMalloc((void **)&s.d_tiles, 2 * sizeof(long long)));
            RC_CK(cudaHostAlloc((void **)&s.h_tiles, 2 * sizeof(long long), cudaHostAllocDefault));
            RC_CK(cudaMalloc((void **)&s.d_counter, sizeof(unsigned long long)));
            RC_CK(cudaMalloc((void **)&s.d_out, sizeof(TallyOut)));
            RC_CK(cudaHostAlloc((void **)&s.h_out, sizeof(TallyOut), cudaHostAllocDefault));
            RC_CK(cudaMalloc((void **)&s.d_desc, sizeof(DSolve<R>)));
            RC_CK(cudaHostAlloc((void **)&s.h_desc, sizeof(DSolve<R>), cudaHostAllocDefault));
            // multigrid pyramid and wall emission arrays
            s.d_levT.assign(nl, nullptr);
            {
                long long tot = 0;
                for (int l = 0; l < nl; ++l) tot += (long long)p.maxi[l] * p.maxj[l] * p.maxk[l];
                RC_CK(cudaMalloc((void **)&s.d_levAll, tot * sizeof(uint16_t)));
                RC_CK(cudaMemset(s.d_levAll, 0, tot * sizeof(uint16_t)));
                for (int l = 0; l < nl; ++l) s.d_levT[l] = s.d_levAll + lev_off[l];
            }
            LevelJobs &J = s.jobs;
            memset(&J, 0, sizeof(J));
            auto add_job = [&](void *dst, int type, int l, int face, long long n) {
                LevelJob &jb = J.job[J.njobs++];
                jb.dst = dst;
                jb.type = type;
                jb.im = p.maxi[l];
                jb.jm = p.maxj[l];
                jb.km = p.maxk[l];
                jb.rx = p.imax / p.maxi[l];
                jb.ry = p.jmax / p.maxj[l];
                jb.rz = p.kmax / p.maxk[l];
                jb.face = face;
                jb.n = n;
                jb.start = J.total;
                J.total += n;
            };
            for (int l = 0; l < nl; ++l) {
                const long long n = (long long)p.maxi[l] * p.maxj[l] * p.maxk[l];
                add_job(s.d_levT[l], 0, l, 0, n);
                for (int w = 0; w < 6; ++w) {
                    const int t = c->wt[w];
                    if (t != WT_BLACK_CELL && t != WT_BLACK_FACE) continue;
                    long long n2;
                    if (w <= RC_EAST) n2 = (long long)p.maxj[l] * p.maxk[l];
                    else if (w <= RC_NORTH) n2 = (long long)p.maxi[l] * p.maxk[l];
                    else n2 = (long long)p.maxi[l] * p.maxj[l];
                    RC_CK(cudaMalloc((void **)&s.d_lw[l][w], n2 * sizeof(uint16_t)));
                    add_job(s.d_lw[l][w], 1 + w, l, t == WT_BLACK_FACE ? 1 : 0, n2);
                }
            }
            // level-0 x-face temperatures: emission temperature of the
            // wall kernel (kernel_surface :1359-1366)
            for (int b = 0; b < 2; ++b) {
                const long long n2 = (long long)p.jmax * p.kmax;
                RC_CK(cudaMalloc((void **)&s.d_Tw0[b], n2 * sizeof(uint16_t)));
                add_job(s.d_Tw0[b], 1 + b, 0, 1, n2);
            }
            const int nBmax = p.grey ? p.grey_nB : p.nB;
            RC_CK(cudaMalloc((void **)&s.d_cdf_f, nBmax * sizeof(R)));
            RC_CK(cudaMalloc((void **)&s.d_cdf_s, nBmax * sizeof(R)));
            const int nQmax = p.grey ? 1 : p.nQ;
            RC_CK(cudaMalloc((void **)&s.d_den_f, (size_t)nBmax * nQmax * sizeof(R)));
            RC_CK(cudaMalloc((void **)&s.d_ibm, nBmax * sizeof(R)));
            RC_CK(cudaMalloc((void **)&s.d_guide_f, kGuide * sizeof(int)));
            RC_CK(cudaMalloc((void **)&s.d_guide_s, kGuide * sizeof(int)));
            RC_CK(cudaMemset(s.d_guide_s, 0, kGuide * sizeof(int)));
            if (p.grey) {
                RC_CK(cudaMalloc((void **)&s.d_Tnb_grey, p.grey_nT * sizeof(R)));
                RC_CK(cudaMalloc((void **)&s.d_Ibt_grey, (size_t)p.grey_nT * p.grey_nB * sizeof(R)));
                RC_CK(cudaMalloc((void **)&s.d_ki_grey, (size_t)p.grey_nT * p.grey_nB * sizeof(KIRow<R>)));
            }
        }
        cudaDeviceProp prop;
        RC_CK(cudaGetDeviceProperties(&prop, c->device));
        c->num_sms = prop.multiProcessorCount;
        smem_opt_in = (int)prop.sharedMemPerBlockOptin;
        RC_CK(cudaFuncSetAttribute(k_march<R, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        if (p.grey) return set_grey_tables();
        return RC_OK;
    }

    // Grey gas: 1000 bands of 5 cm^-1 up to wvmax with k = abscoeff
    // (read_tables.cpp:98-137); the Planck table and band CDF depend on
    // Tmax and are rebuilt on the device by every solve.
    int set_grey_tables() {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        release_tables();
        nT = p.grey_nT;
        nB = p.grey_nB;
        nQ = 1;
        std::vector<float> wvl(nB), wvr(nB), wvc(nB);
        const float dw = p.wvmax / nB;
        wvl[0] = 0;
        for (int i = 1; i < nB; i++) wvl[i] = wvl[i - 1] + dw;
        wvr[0] = dw;
        for (int i = 1; i < nB; i++) wvr[i] = wvr[i - 1] + dw;
        for (int i = 0; i < nB; i++) wvc[i] = (float)((double)(wvl[i] + wvr[i]) / 2.);
        std::vector<float> kt((size_t)nB * nT, p.abscoeff), kP(nT, p.abscoeff), probq(1, 1.0f);
        std::vector<float> probg((size_t)nT * nB, 1.0f);
        std::vector<float> Ibw((size_t)6 * nB);
        for (int w = 0; w < 6; ++w)
            for (int b = 0; b < nB; ++b) Ibw[(size_t)w * nB + b] = (float)rc_planck((double)p.Tw[w], (double)wvc[b]);
        int rc = upload(d_kt, kt, err_);
        if (!rc) rc = upload(d_kP, kP, err_);
        if (!rc) rc = upload(d_probq, probq, err_);
        if (!rc) rc = upload(d_probg, probg, err_);
        if (!rc) rc = upload(d_Ibw, Ibw, err_);
        if (!rc) rc = upload(d_wvl, wvl, err_);
        if (!rc) rc = upload(d_wvr, wvr, err_);
        if (!rc) rc = upload(d_wvc, wvc, err_);
        if (rc) return rc;
        c->has_tables = true;
        c->gen++;
        return RC_OK;
    }

    int set_tables(const TableSet &t) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        if (p.grey) return set_err(err_, RC_E_INVALID, "grey mode builds its own tables; rc_set_tables not used");
        if (t.nT != p.nT || t.nB != p.nB || t.nQ != p.nQ)
            return set_err(err_, RC_E_INVALID, "table dimensions differ from params nT/nB/nQ");
        {
            std::string m;
            if (tables_check(t, m)) return set_err(err_, RC_E_INVALID, m);
        }
        release_tables();
        nT = t.nT;
        nB = t.nB;
        nQ = t.nQ;
        const float ch = (float)p.chanHeight;
        // k scaled by chanHeight (read_tables.cpp:30,56), stored [nB][nQ][nT]
        std::vector<float> kt((size_t)nB * nQ * nT), kP(nT), Ibt((size_t)nB * nT);
        for (int b = 0; b < nB; ++b)
            for (int g = 0; g < nQ; ++g)
                for (int i = 0; i < nT; ++i) {
                    float k = t.kq[((size_t)b * nT + i) * nQ + g];
                    k = (float)((double)k * p.chanHeight);
                    kt[((size_t)b * nQ + g) * nT + i] = k;
                }
        for (int i = 0; i < nT; ++i) kP[i] = (float)((double)t.kP[i] * p.chanHeight);
        (void)ch;
        // Planck table Ib[nb][t] = I_blackC(Tnb[t], wvc[nb]) (mc_gpu_noint.cu:770-780)
        for (int b = 0; b < nB; ++b)
            for (int i = 0; i < nT; ++i) Ibt[(size_t)b * nT + i] = (float)rc_planck((double)t.Tnb[i], (double)t.wvc[b]);
        std::vector<float> Ibw((size_t)6 * nB);
        for (int w = 0; w < 6; ++w)
            for (int b = 0; b < nB; ++b) Ibw[(size_t)w * nB + b] = (float)rc_planck((double)p.Tw[w], (double)t.wvc[b]);
        // wall g CDF: cumulative g weights (mc_gpu_noint.cu:34-36), last = 1
        std::vector<float> probq(nQ);
        float cq = 0.f;
        for (int g = 0; g < nQ; ++g) {
            cq += t.wq[g];
            probq[g] = (g == nQ - 1) ? 1.0f : cq;
        }
        int rc = upload(d_kt, kt, err_);
        if (!rc) rc = upload(d_kP, kP, err_);
        if (!rc) rc = upload(d_Ibt, Ibt, err_);
        if (!rc) rc = upload(d_Ibw, Ibw, err_);
        if (!rc) rc = upload(d_probq, probq, err_);
        if (!rc) rc = upload(d_prob, t.prob, err_);
        if (!rc) rc = upload(d_probg, t.probg, err_);
        if (!rc) rc = upload(d_Tnb, t.Tnb, err_);
        if (!rc) rc = upload(d_wvl, t.wvl, err_);
        if (!rc) rc = upload(d_wvr, t.wvr, err_);
        if (!rc) rc = upload(d_wvc, t.wvc, err_);
        if (rc) return rc;
        // interleaved rows {k[t], Ib[t], k[t+1], Ib[t+1]} for the march
        std::vector<KIRow<R>> ki((size_t)nB * nQ * nT);
        for (int b = 0; b < nB; ++b)
            for (int g = 0; g < nQ; ++g)
                for (int i = 0; i < nT; ++i) {
                    const int i1 = std::min(i + 1, nT - 1);
                    KIRow<R> &r = ki[((size_t)b * nQ + g) * nT + i];
                    r.k0 = (R)kt[((size_t)b * nQ + g) * nT + i];
                    r.k1 = (R)kt[((size_t)b * nQ + g) * nT + i1];
                    r.ib0 = (R)Ibt[(size_t)b * nT + i];
                    r.ib1 = (R)Ibt[(size_t)b * nT + i1];
                }
        RC_CK(cudaMalloc((void **)&d_ki, ki.size() * sizeof(KIRow<R>)));
        RC_CK(cudaMemcpy(d_ki, ki.data(), ki.size() * sizeof(KIRow<R>), cudaMemcpyHostToDevice));
        c->has_tables = true;
        c->gen++;
        return RC_OK;
    }

    // Scattering particles for later solves (nullptr: none).  The table
    // must match the context's bands and g points (grey: grey_nB bands, one
    // g point).  ksca is scaled by chanHeight like k (read_tables.cpp:30,56);
    // angles become turns (theta / 2 pi), the argument of the march's
    // sin/cos; the last CDF entry of every band is set to exactly 1.
    int set_scattering(const rc_scattering *s) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        if (!s) {
            RC_CK(cudaDeviceSynchronize());
            release_scattering();
            c->gen++;
            return RC_OK;
        }
        const int nBc = p.grey ? p.grey_nB : p.nB, nQc = p.grey ? 1 : p.nQ;
        if (s->nB != nBc || s->nQ != nQc)
            return set_err(err_, RC_E_INVALID, "scattering table bands / g points differ from the context's");
        {
            char msg[256];
            if (rc_scattering_validate(s, msg, sizeof(msg))) return set_err(err_, RC_E_INVALID, msg);
        }
        // a kernel still reading the old arrays (a solve or batch of this
        // context) finishes before they are freed
        RC_CK(cudaDeviceSynchronize());
        std::vector<float> ks((size_t)s->nB * s->nQ), cdf((size_t)s->nB * s->nA), th(s->nA);
        for (size_t i = 0; i < ks.size(); ++i) ks[i] = rc_scatter_coef_scaled(s->ksca[i], p.chanHeight);
        for (int b = 0; b < s->nB; ++b)
            for (int a = 0; a < s->nA; ++a)
                cdf[(size_t)b * s->nA + a] = (a == s->nA - 1) ? 1.0f : s->phase_cdf[(size_t)b * s->nA + a];
        for (int a = 0; a < s->nA; ++a) th[a] = rc_angle_turns(s->theta[a]);
        // search brackets of the phase CDF (phase_index): guide[q] is the
        // first angle a >= 1 with cdf[a] > q / kPhaseGuide, nA-1 if none
        std::vector<uint16_t> guide((size_t)s->nB * (kPhaseGuide + 1));
        for (int b = 0; b < s->nB; ++b) {
            const float *cb = &cdf[(size_t)b * s->nA];
            int a = 1;
            for (int q = 0; q <= kPhaseGuide; ++q) {
                const float thr = (float)q / (float)kPhaseGuide;
                while (a < s->nA - 1 && !(cb[a] > thr)) ++a;
                guide[(size_t)b * (kPhaseGuide + 1) + q] = (uint16_t)a;
            }
        }
        release_scattering();
        int rc = upload(d_ksca, ks, err_);
        if (!rc) rc = upload(d_pcdf, cdf, err_);
        if (!rc) rc = upload(d_pth, th, err_);
        if (!rc) {
            cudaError_t e = cudaMalloc((void **)&d_pguide, guide.size() * sizeof(uint16_t));
            if (e == cudaSuccess)
                e = cudaMemcpy(d_pguide, guide.data(), guide.size() * sizeof(uint16_t), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) rc = set_err(err_, RC_E_CUDA, std::string("phase guide: ") + cudaGetErrorString(e));
        }
        if (rc) {
            release_scattering();
            return rc;
        }
        nA = s->nA;
        c->gen++;
        return RC_OK;
    }

    // Work decomposition: items of rpt bundles, chunk count padded so that
    // the chunks of one (cell, replicate) never straddle a 32-item tile.
    void decompose(int rpt, int &nchunk, int &gsize, int &nparts, int photmax = 0) const {
        if (photmax <= 0) photmax = c->p.photmax;
        int nc = (photmax + rpt - 1) / rpt;
        if (nc <= kWarp) {
            int p2 = 1;
            while (p2 < nc) p2 <<= 1;
            nc = p2;
            gsize = nc;
            nparts = 1;
        } else {
            nc = (nc + kWarp - 1) / kWarp * kWarp;
            gsize = kWarp;
            nparts = nc / kWarp;
        }
        nchunk = nc;
    }

    void fill_desc(Slot<R> &s, int zstart, int rpt, DSolve<R> &d) {
        const rc_params &p = c->p;
        memset(&d, 0, sizeof(d));
        d.nlev = p.grid_num;
        for (int l = 0; l < p.grid_num; ++l) {
            DLevel<R> &L = d.lev[l];
            L.im = p.maxi[l];
            L.jm = p.maxj[l];
            L.km = p.maxk[l];
            L.maxs = p.maxs[l];
            if (l + 1 < p.grid_num) {
                L.rx = p.maxi[l] / p.maxi[l + 1];
                L.ry = p.maxj[l] / p.maxj[l + 1];
                L.rz = p.maxk[l] / p.maxk[l + 1];
            } else {
                L.rx = L.ry = L.rz = 1;
            }
            L.mrx = magic32(L.rx);
            L.mry = magic32(L.ry);
            L.mrz = magic32(L.rz);
            L.xu = d_xu[l];
            L.yu = d_yu[l];
            L.zu = d_zu[l];
            L.P = s.d_levT[l];
            d.lva[l] = make_int4(face_off[l], face_off[l] + L.im + 1, face_off[l] + L.im + 1 + L.jm + 1, lev_off[l]);
            d.lvb[l] = make_int4(L.im, L.jm, L.km, L.maxs);
            for (int w = 0; w < 6; ++w) L.Pw[w] = s.d_lw[l][w];
        }
        d.imax = p.imax;
        d.jmax = p.jmax;
        d.kmax = p.kmax;
        d.kloc = c->kloc;
        d.kfirst = zstart;
        for (int w = 0; w < 6; ++w) d.wtype[w] = c->wt[w];
        d.nT = nT;
        d.nB = nB;
        d.nQ = nQ;
        d.nVar = p.nVar;
        d.photmax = p.photmax;
        d.rpt = rpt;
        d.sort = c->sort ? 1 : 0;
        decompose(rpt, d.nchunk, d.gsize, d.nparts);
        d.nwalls = 0;
        if (p.calcwalls) {
            if (p.adiabw) d.wall_id[d.nwalls++] = 0;
            if (p.adiabe) d.wall_id[d.nwalls++] = 1;
        }
        d.Lx = (R)p.Lx;
        d.Ly = (R)p.Ly;
        d.Lz = (R)p.Lz;
        d.toll = (R)p.toll;
        d.tollS = (R)p.tollS;
        d.faces = d_faces;
        d.Pall = s.d_levAll;
        d.xc = d_xc;
        d.yc = d_yc;
        d.zc = d_zc;
        d.kt = d_kt;
        d.Ibt = p.grey ? s.d_Ibt_grey : d_Ibt;
        d.probg = d_probg;
        d.cdf_f = s.d_cdf_f;
        d.cdf_s = s.d_cdf_s;
        d.den_f = s.d_den_f;
        d.ibm = s.d_ibm;
        d.guide_f = s.d_guide_f;
        d.guide_s = s.d_guide_s;
        d.ksca = d_ksca;
        d.pcdf = d_pcdf;
        d.pth = d_pth;
        d.pguide = d_pguide;
        d.nA = nA;
        d.probq = d_probq;
        d.Ibw = d_Ibw;
        d.Pw0[0] = s.d_Tw0[0];
        d.Pw0[1] = s.d_Tw0[1];
        d.ki = p.grey ? s.d_ki_grey : d_ki;
        d.sc = s.d_sc;
        d.partial = s.d_partial;
        d.n_faces = n_faces;
        d.n_P = n_pyramid;
        d.n_partial = (long long)partial_count(rpt);
        const long long ncf = (long long)p.imax * p.jmax * c->kloc;
        d.n_fluid_items = ncf * p.nVar * d.nchunk;
        d.n_items = d.n_fluid_items + (long long)d.nwalls * p.jmax * c->kloc * p.nVar * d.nchunk;
        d.n_tiles = (d.n_items + kWarp - 1) / kWarp;
        d.key0 = (uint32_t)p.seed;
        d.key1 = (uint32_t)(p.seed >> 32);
        d.tile_base = 0;
        d.nwc = (unsigned long long)p.jmax * c->kloc;
        d.mg_nchunk = magic(d.nchunk);
        d.mg_nvar = magic(p.nVar);
        d.mg_imax = magic(p.imax);
        d.mg_jmax = magic(p.jmax);
        d.mg_nwc = magic(d.nwc);
    }

    // Multiply-high reciprocal of a divisor d (see fdiv): floor((2^64-1)/d)+1,
    // 0 for d = 1.
    static unsigned long long magic(unsigned long long d) {
        return d <= 1 ? 0ull : (~0ull / d) + 1ull;
    }
    static unsigned magic32(unsigned d) { return d <= 1 ? 0u : (unsigned)(0xffffffffu / d) + 1u; }

    // fdiv is exact when numerator * divisor < 2^64 at every division of the
    // item decomposition.
    bool decomposition_fits(const DSolve<R> &d) const {
        const long double lim = 18446744073709551615.0L;
        const long double n = (long double)d.n_items;
        bool ok = n * d.nchunk < lim && n * d.nVar < lim && n * c->p.imax < lim && n * c->p.jmax < lim &&
                  n * (long double)d.nwc < lim;
        // coarse_index is exact when (n + r - 1) * r < 2^32 on every axis
        for (int l = 0; l + 1 < d.nlev; ++l) {
            const DLevel<R> &L = d.lev[l];
            ok = ok && (double)(L.im + L.rx) * L.rx < 4294967296.0 && (double)(L.jm + L.ry) * L.ry < 4294967296.0 &&
                 (double)(L.km + L.rz) * L.rz < 4294967296.0;
        }
        return ok;
    }

    size_t partial_count(int rpt, int photmax = 0) const {
        int nchunk, gsize, nparts;
        decompose(rpt, nchunk, gsize, nparts, photmax);
        const rc_params &p = c->p;
        const long long ncells = (long long)p.imax * p.jmax * c->kloc + 2LL * p.jmax * c->kloc;
        return (size_t)ncells * p.nVar * nparts;
    }

    int ensure_partial(Slot<R> &s, int rpt) {
        std::string *err_ = &c->err;
        const size_t need = partial_count(rpt);
        if (need > s.partial_cap) {
            if (s.d_partial) {
                RC_CK(cudaStreamSynchronize(s.st));
                cudaFree(s.d_partial);
                s.d_partial = nullptr;
            }
            RC_CK(cudaMalloc((void **)&s.d_partial, need * sizeof(double)));
            s.partial_cap = need;
        }
        return RC_OK;
    }

    // Set-up kernels of one solve (everything before the march).
    int enqueue_setup(Slot<R> &s, cudaStream_t st) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        k_init_scalars<<<1, 32, 0, st>>>(s.d_sc);
        const long long ncell = (long long)p.imax * p.jmax * p.kmax;
        int gb = (int)std::min<long long>((ncell + 255) / 256, (long long)c->num_sms * 8);
        k_tmax<<<std::max(gb, 1), 256, 0, st>>>(s.d_T, p.imax, p.jmax, p.kmax, s.d_sc);
        R *Tnb = p.grey ? s.d_Tnb_grey : d_Tnb;
        k_setup1<R><<<1, 32, 0, st>>>(s.d_sc, Tnb, d_kP, nT, p.grey, p.Tmins, p.abscoeff, p.stefan, p.photmax,
                                      p.eps[RC_WEST], p.eps[RC_EAST]);
        const R *Ibt = d_Ibt;
        if (p.grey) {
            const int n = nT * nB;
            k_grey_ib<R><<<std::max(1, std::min((n + 255) / 256, c->num_sms * 4)), 256, 0, st>>>(s.d_Ibt_grey, Tnb,
                                                                                                  d_wvc, nT, nB);
            Ibt = s.d_Ibt_grey;
            k_build_ki<R><<<std::max(1, std::min((n + 255) / 256, c->num_sms * 4)), 256, 0, st>>>(s.d_ki_grey, d_kt,
                                                                                                Ibt, nB, 1, nT);
        }
        k_setup2<R><<<1, 256, 0, st>>>(s.d_sc, s.d_cdf_f, s.d_cdf_s, s.d_guide_f, s.d_guide_s, s.d_den_f, s.d_ibm,
                                       d_prob, Ibt, d_kt, d_wvl, d_wvr, nT, nB, nQ, p.grey, p.calcwalls);
        const LevelJobs &J = s.jobs;
        int gl = (int)std::min<long long>((J.total + 255) / 256, (long long)c->num_sms * 8);
        k_levels<R><<<std::max(gl, 1), 256, 0, st>>>(s.d_T, p.imax, p.jmax, p.kmax, J, s.d_sc, nT);
        RC_CK(cudaGetLastError());
        return RC_OK;
    }

    size_t march_smem(int block, int rpt_max, bool scat = false) const {
        return scat ? march_smem_bytes<R, true>(block, rpt_max) : march_smem_bytes<R, false>(block, rpt_max);
    }

    static void (*march_fn(int minb, bool scat))(MarchArgs) {
        if (scat) return minb <= 2 ? k_march<R, 2, true> : minb == 3 ? k_march<R, 3, true> : k_march<R, 4, true>;
        return minb <= 2 ? k_march<R, 2, false> : minb == 3 ? k_march<R, 3, false> : k_march<R, 4, false>;
    }

    // Long-ray priority list of a one-solve launch (k_prio_kmin +
    // k_prio_tiles) on stream st, into the slot's buffers; `use` stays false
    // when the knob is off or the solve has more tiles than the list is kept
    // for (its tail is then a small share of the launch).  The list is built
    // from the bundles' own draws, band CDF and temperature range of the
    // solve it is first built for, and kept while the draws and the work
    // decomposition stay the same (seed, photmax, rays_per_thread,
    // replicates, grid, walls, threshold): a DNS calling with one parameter
    // set every radStep pays for it once, and a later field can only make the
    // order less apt, never change a result.  The tail it removes is a fixed
    // few ms per launch (the longest rays), while reordering costs pyramid
    // locality in proportion to the work, hence the limit on tiles.
    static constexpr long long kPrioMaxTiles = 1LL << 22;
    int enqueue_prio(Slot<R> &s, cudaStream_t st, bool &use) {
        std::string *err_ = &c->err;
        use = false;
        const DSolve<R> &d = *s.h_desc;
        const long long nt = d.n_tiles;
        if (!(c->prio_thr > 0.f) || nt < 1 || nt > kPrioMaxTiles) return RC_OK;
        unsigned thr_bits;
        memcpy(&thr_bits, &c->prio_thr, 4);
        const long long key[10] = {(long long)d.key0 | ((long long)d.key1 << 32), d.photmax, d.rpt, d.nVar,
                                   (long long)d.imax | ((long long)d.jmax << 32),
                                   (long long)d.kloc | ((long long)d.kfirst << 32), nt,
                                   (long long)d.nwalls | ((long long)d.wall_id[0] << 8) | ((long long)d.wall_id[1] << 16),
                                   (long long)thr_bits, (long long)sizeof(R)};
        if (s.prio_ok && s.prio_cap >= nt && memcmp(key, s.prio_key, sizeof(key)) == 0) {
            use = true;
            return RC_OK;
        }
        s.prio_ok = false;
        if (s.prio_cap < nt) {
            dfree(s.d_prio);
            dfree(s.d_tprio);
            s.prio_cap = 0;
            RC_CK(cudaMalloc((void **)&s.d_prio, nt * sizeof(unsigned)));
            RC_CK(cudaMalloc((void **)&s.d_tprio, nt));
            s.prio_cap = nt;
        }
        const int nbq = d.nB * d.nQ;
        if (s.kmin_cap < nbq) {
            dfree(s.d_kmin);
            s.kmin_cap = 0;
            RC_CK(cudaMalloc((void **)&s.d_kmin, nbq * sizeof(float)));
            s.kmin_cap = nbq;
        }
        if (!s.d_nprio) RC_CK(cudaMalloc((void **)&s.d_nprio, sizeof(unsigned)));
        RC_CK(cudaMemsetAsync(s.d_nprio, 0, sizeof(unsigned), st));
        k_prio_kmin<R><<<(nbq + 255) / 256, 256, 0, st>>>(s.d_desc, s.d_kmin);
        RC_CK(cudaGetLastError());
        const long long grid = std::max<long long>(1, std::min<long long>((nt + 7) / 8, (long long)c->num_sms * 16));
        k_prio_tiles<R><<<(unsigned)grid, 256, 0, st>>>(s.d_desc, c->prio_thr, s.d_kmin, s.d_prio, s.d_tprio,
                                                         s.d_nprio);
        RC_CK(cudaGetLastError());
        memcpy(s.prio_key, key, sizeof(key));
        s.prio_ok = true;
        use = true;
        return RC_OK;
    }

    // scat: < 0 takes this context's medium (scattering tables set or not);
    // a launch over several contexts passes whether any of them scatters.
    int launch_march(const DSolve<R> *d_solves, const long long *d_tiles, int nsolves, long long total_tiles,
                     unsigned long long *d_counter, int block, int rpt_max, cudaStream_t st, int minb = 0,
                     const Slot<R> *prio = nullptr, int scat = -1) {
        std::string *err_ = &c->err;
        RC_FAILPOINT("march");
        if (minb <= 0) minb = c->minb;
        const bool sc = scat < 0 ? nA > 0 : scat > 0;
        auto fn = march_fn(minb, sc);
        const size_t smem = march_smem(block, rpt_max, sc);
        if ((int)smem > smem_opt_in) return set_err(err_, RC_E_INVALID, "rays_per_thread too large for shared memory");
        int per_sm = 0;
        RC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
        per_sm = std::max(per_sm, 1);
        const long long warps_needed = total_tiles;
        long long grid = std::min<long long>((long long)per_sm * c->num_sms, (warps_needed + block / kWarp - 1) / (block / kWarp));
        grid = std::max<long long>(grid, 1);
        RC_CK(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), st));
        MarchArgs a;
        a.solves = d_solves;
        a.tile_start = d_tiles;
        a.nsolves = nsolves;
        a.total_tiles = total_tiles;
        a.tile_counter = d_counter;
        a.rpt_max = rpt_max;
        a.prio_tiles = prio ? prio->d_prio : nullptr;
        a.tile_prio = prio ? prio->d_tprio : nullptr;
        a.n_prio = prio ? prio->d_nprio : nullptr;
        fn<<<(unsigned)grid, block, smem, st>>>(a);
        RC_CK(cudaGetLastError());
        return RC_OK;
    }

    Slot<R> *find_slot(rc_ticket t) {
        for (auto &s : slots)
            if (s.ticket == t && s.state != 0) return &s;
        return nullptr;
    }

    Slot<R> *free_slot() {
        for (auto &s : slots)
            if (s.state == 0) return &s;
        return nullptr;
    }

    int check_solve_args(const float *T, int zstart) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        if (!c->has_tables) return set_err(err_, RC_E_STATE, "no tables: call rc_set_tables first");
        if (!T) return set_err(err_, RC_E_INVALID, "T is NULL");
        if (zstart < 1 || zstart + c->kloc - 1 > p.kmax) return set_err(err_, RC_E_INVALID, "zstart out of range");
        return RC_OK;
    }

    // Stage the field into the slot's pinned buffer (the caller's array is
    // copied before return, as mc_gpu_noint.cu:676-690 does).
    int stage_host_field(Slot<R> &s, const float *T) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        const size_t nfield = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
        RC_CK(cudaStreamSynchronize(s.st));
        memcpy(s.h_T, T, nfield * sizeof(float));
        return RC_OK;
    }

    // Host half of a solve's preparation: the descriptor (s.h_desc) and the
    // tally outputs (s.h_out); no device work.
    int prepare_host(Slot<R> &s, int zstart, int rpt) {
        std::string *err_ = &c->err;
        int rc = ensure_partial(s, rpt);
        if (rc) return rc;
        fill_desc(s, zstart, rpt, *s.h_desc);
        if (!decomposition_fits(*s.h_desc))
            return set_err(err_, RC_E_INVALID, "too many work items for one solve: raise rays_per_thread");
        TallyOut *o = s.h_out;
        o->q64 = s.d_q64;
        o->var64 = s.d_var64;
        o->qw64 = s.d_qw64;
        o->vw64 = s.d_vw64;
        o->Qc = s.d_Qc;
        o->Sc = s.d_Sc;
        o->Wq = s.d_Wq;
        o->Ws = s.d_Ws;
        s.zstart = zstart;
        s.rpt = rpt;
        return RC_OK;
    }

    // Device half on stream st: the field copy (from T_dev, else from the
    // slot's pinned staging; none when the caller has filled s.d_T), the
    // set-up kernels, and the descriptor at desc_dev patched with the run-time
    // scalars.  A batch passes its own descriptor array, already copied from
    // the members' s.h_desc; a single solve the slot's (copied here, with the
    // tally outputs).
    int prepare_device(Slot<R> &s, const float *T_dev, bool field_ready, DSolve<R> *desc_dev, cudaStream_t st) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        RC_FAILPOINT("field_copy");
        const size_t nfield = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
        if (T_dev) RC_CK(cudaMemcpyAsync(s.d_T, T_dev, nfield * sizeof(float), cudaMemcpyDeviceToDevice, st));
        else if (!field_ready) RC_CK(cudaMemcpyAsync(s.d_T, s.h_T, nfield * sizeof(float), cudaMemcpyHostToDevice, st));
        int rc = enqueue_setup(s, st);
        if (rc) return rc;
        if (desc_dev == s.d_desc) {
            RC_CK(cudaMemcpyAsync(s.d_desc, s.h_desc, sizeof(DSolve<R>), cudaMemcpyHostToDevice, st));
            RC_CK(cudaMemcpyAsync(s.d_out, s.h_out, sizeof(TallyOut), cudaMemcpyHostToDevice, st));
        }
        k_patch_desc<R><<<1, 32, 0, st>>>(desc_dev, s.d_sc);
        RC_CK(cudaGetLastError());
        return RC_OK;
    }

    // Everything up to the march on stream st: field copy, set-up kernels
    // and the descriptor (built into s.h_desc, copied to s.d_desc).
    int prepare(Slot<R> &s, const float *T_dev, int zstart, int rpt, cudaStream_t st) {
        int rc = prepare_host(s, zstart, rpt);
        if (rc) return rc;
        return prepare_device(s, T_dev, false, s.d_desc, st);
    }

    size_t field_floats() const {
        const rc_params &p = c->p;
        return (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
    }

    int launch_tally(const DSolve<R> *d_solves, const TallyOut *d_outs, int nsolves, long long max_cells,
                     cudaStream_t st) {
        std::string *err_ = &c->err;
        RC_FAILPOINT("tally");
        const int gt = (int)std::max<long long>(1, std::min<long long>((max_cells + 255) / 256, (long long)c->num_sms * 8));
        k_tally_multi<R><<<dim3(gt, nsolves), 256, 0, st>>>(d_solves, d_outs);
        RC_CK(cudaGetLastError());
        return RC_OK;
    }

    long long tally_cells() const {
        const rc_params &p = c->p;
        return (long long)p.imax * p.jmax * c->kloc + 2LL * p.jmax * c->kloc;
    }

    int solve(const float *T, bool device_ptr, int zstart, rc_ticket *ticket) {
        Range nv("rc_solve");
        std::string *err_ = &c->err;
        int rc = check_solve_args(T, zstart);
        if (rc) return rc;
        Slot<R> *sp = free_slot();
        if (!sp) return set_err(err_, RC_E_BUSY, "all solve slots in use: collect a ticket first");
        Slot<R> &s = *sp;
        const int rpt = c->rpt;
        if (!device_ptr) {
            rc = stage_host_field(s, T);
            if (rc) return rc;
        }
        RC_CK(cudaEventRecord(s.e0, s.st));
        rc = prepare(s, device_ptr ? T : nullptr, zstart, rpt, s.st);
        if (rc) return rc;
        s.h_tiles[0] = 0;
        s.h_tiles[1] = s.h_desc->n_tiles;
        RC_CK(cudaMemcpyAsync(s.d_tiles, s.h_tiles, 2 * sizeof(long long), cudaMemcpyHostToDevice, s.st));
        // the long-ray priority list (built once per slot, then reused):
        // also while the other slot's solve runs, where it measured 28.1 ms
        // per solve end to end against 28.8-29.1 ms without it
        RC_CK(cudaEventRecord(s.e_march0, s.st));
        bool prio = false;
        rc = enqueue_prio(s, s.st, prio);
        if (rc) return rc;
        rc = launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, c->block, rpt, s.st, 0,
                          prio ? &s : nullptr);
        if (rc) return rc;
        RC_CK(cudaEventRecord(s.e_march1, s.st));
        rc = launch_tally(s.d_desc, s.d_out, 1, tally_cells(), s.st);
        if (rc) return rc;
        RC_CK(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(DScalars), cudaMemcpyDeviceToHost, s.st));
        RC_CK(cudaEventRecord(s.e1, s.st));
        s.state = 1;
        s.ticket = c->next_ticket++;
        s.block = c->block;
        s.host_copied = false;
        *ticket = s.ticket;
        return RC_OK;
    }

    // Launch-configuration sweep on a reduced bundle count: the knobs do
    // not change the sampled bundles (counter-based draws), only the work
    // decomposition, the FP64 summation grouping and the order in which a
    // warp's lanes take bundles.
    // March time of one launch configuration on the pilot: the best of two
    // timed launches after a warm-up launch.
    int time_config(Slot<R> &s, int zstart, int rpt, int block, int minb, float *ms_out) {
        std::string *err_ = &c->err;
        float tot = 3.4e38f;
        for (int rep = 0; rep < 3; ++rep) {
            int rc = prepare(s, nullptr, zstart, rpt, s.st);
            if (rc) return rc;
            s.h_tiles[0] = 0;
            s.h_tiles[1] = s.h_desc->n_tiles;
            RC_CK(cudaMemcpyAsync(s.d_tiles, s.h_tiles, 2 * sizeof(long long), cudaMemcpyHostToDevice, s.st));
            RC_CK(cudaEventRecord(s.e_march0, s.st));
            bool prio = false;
            rc = enqueue_prio(s, s.st, prio);
            if (rc) return rc;
            rc = launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, block, rpt, s.st, minb,
                              prio ? &s : nullptr);
            if (rc) return rc;
            RC_CK(cudaEventRecord(s.e_march1, s.st));
            RC_CK(cudaEventSynchronize(s.e_march1));
            float ms = 0.f;
            RC_CK(cudaEventElapsedTime(&ms, s.e_march0, s.e_march1));
            if (rep > 0) tot = std::min(tot, ms);  // the first run warms up
        }
        *ms_out = tot;
        return RC_OK;
    }

    int autotune(const float *T, int zstart, int pilot, int *rpt_out, int *block_out, int *sort_out, int *occ_out) {
        Range nv("rc_autotune");
        std::string *err_ = &c->err;
        int rc = check_solve_args(T, zstart);
        if (rc) return rc;
        Slot<R> *sp = free_slot();
        if (!sp) return set_err(err_, RC_E_BUSY, "all solve slots in use");
        Slot<R> &s = *sp;
        const int saved_photmax = c->p.photmax, saved_sort = c->sort;
        // the pilot is raised until its launch has 10^8 bundles or more
        // (at most the real photmax): a shorter launch is dominated by its
        // tail and launch latency, and ranks configurations by those
        {
            const rc_params &p = c->p;
            const long long cellsv =
                ((long long)p.imax * p.jmax * c->kloc + 2LL * p.jmax * c->kloc) * std::max(p.nVar, 1);
            int pp = pilot > 0 ? std::min(pilot, saved_photmax) : saved_photmax;
            while ((long long)pp * cellsv < 100000000LL && pp < saved_photmax) pp = std::min(2 * pp, saved_photmax);
            c->p.photmax = pp;
        }
        const int p1 = c->p.photmax;
        rc = stage_host_field(s, T);
        // Estimated time of the real solve.  A pilot's launch carries a tail
        // (its last, longest rays) that a long solve hides, so a pilot much
        // smaller than the real photmax is timed at p1 and 2 p1 bundles per
        // cell: t(P) = t(p1) + (t(2 p1) - t(p1)) (P - p1) / p1, the marginal
        // cost per bundle carrying the estimate.  Writing and reading the FP64
        // partial sums that rays_per_thread implies at the real photmax is
        // added.
        const bool two_point = saved_photmax > 4 * p1;
        int mem_khz = 0, bus_bits = 0;
        cudaDeviceGetAttribute(&mem_khz, cudaDevAttrMemoryClockRate, c->device);
        cudaDeviceGetAttribute(&bus_bits, cudaDevAttrGlobalMemoryBusWidth, c->device);
        const double hbm = (mem_khz > 0 && bus_bits > 0) ? 2.0 * mem_khz * 1e3 * bus_bits / 8.0 : 6.5e12;
        auto score = [&](int rpt, int block, int minb, double *est) {
            float t1 = 0.f;
            int r = time_config(s, zstart, rpt, block, minb, &t1);
            if (r) return r;
            double e = (double)t1 * saved_photmax / p1;
            if (two_point) {
                float t2 = 0.f;
                c->p.photmax = 2 * p1;
                r = time_config(s, zstart, rpt, block, minb, &t2);
                c->p.photmax = p1;
                if (r) return r;
                e = (double)t1 + std::max(0.0, (double)t2 - (double)t1) * (double)(saved_photmax - p1) / p1;
            }
            *est = e + 2.0 * 8.0 * (double)partial_count(rpt, saved_photmax) / hbm * 1e3;
            return RC_OK;
        };
        // the current knobs are the incumbent; another configuration must
        // beat it by 3 % to replace it (pilot timings vary by about that)
        c->sort = 0;
        int brpt = c->rpt, bblock = c->block, bminb = c->minb, bsort = 0;
        double best = 1e300;
        if (!rc && march_smem(bblock, brpt, nA > 0) <= (size_t)smem_opt_in) rc = score(brpt, bblock, bminb, &best);
        const int rpts[] = {2, 4, 8, 16, 32};
        const int blocks[] = {128, 256};
        const int minbs[] = {2, 3, 4};
        for (int oi = 0; oi < 3 && !rc; ++oi)
            for (int bi = 0; bi < 2 && !rc; ++bi)
                for (int ri = 0; ri < 5 && !rc; ++ri) {
                    const int rpt = rpts[ri], block = blocks[bi], minb = minbs[oi];
                    if (rpt == brpt && block == bblock && minb == bminb) continue;
                    if (march_smem(block, rpt, nA > 0) > (size_t)smem_opt_in) continue;
                    double e = 0.0;
                    rc = score(rpt, block, minb, &e);
                    if (!rc && e < 0.97 * best) {
                        best = e;
                        brpt = rpt;
                        bblock = block;
                        bminb = minb;
                    }
                }
        if (!rc) {
            c->sort = 1;
            double e = 0.0;
            rc = score(brpt, bblock, bminb, &e);
            if (!rc && e < 0.97 * best) bsort = 1;
        }
        c->p.photmax = saved_photmax;
        if (rc) {
            c->sort = saved_sort;
            return rc;
        }
        c->rpt = brpt;
        c->block = bblock;
        c->minb = bminb;
        c->sort = bsort;
        c->gen++;
        if (rpt_out) *rpt_out = brpt;
        if (block_out) *block_out = bblock;
        if (sort_out) *sort_out = bsort;
        if (occ_out) *occ_out = bminb;
        return RC_OK;
    }

    int wait(Slot<R> &s) {
        std::string *err_ = &c->err;
        RC_CK(cudaEventSynchronize(s.e1));
        s.state = 2;
        return RC_OK;
    }

    int collect(rc_ticket t, float *Q, float *sigma, double *q64, double *var64, double *qw64, double *vw64) {
        Range nv("rc_collect");
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown or already collected ticket");
        Slot<R> &s = *sp;
        int rc = wait(s);
        if (rc) return rc;
        rc = copy_out(s, Q, sigma, q64, var64, qw64, vw64);
        s.state = 0;
        s.ticket = -1;
        return rc;
    }

    // Results of a finished slot to host arrays (synchronous).
    int copy_out(Slot<R> &s, float *Q, float *sigma, double *q64, double *var64, double *qw64, double *vw64) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        RC_FAILPOINT("collect");
        const size_t ncf = (size_t)p.imax * p.jmax * c->kloc;
        const size_t nwc = (size_t)2 * p.jmax * c->kloc;
        if (Q || sigma) {
            RC_CK(cudaMemcpyAsync(s.h_Qc, s.d_Qc, ncf * sizeof(float), cudaMemcpyDeviceToHost, s.st));
            RC_CK(cudaMemcpyAsync(s.h_Sc, s.d_Sc, ncf * sizeof(float), cudaMemcpyDeviceToHost, s.st));
            RC_CK(cudaMemcpyAsync(s.h_Wq, s.d_Wq, nwc * sizeof(float), cudaMemcpyDeviceToHost, s.st));
            RC_CK(cudaMemcpyAsync(s.h_Ws, s.d_Ws, nwc * sizeof(float), cudaMemcpyDeviceToHost, s.st));
        }
        if (q64) RC_CK(cudaMemcpyAsync(q64, s.d_q64, ncf * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        if (var64) RC_CK(cudaMemcpyAsync(var64, s.d_var64, ncf * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        if (qw64) RC_CK(cudaMemcpyAsync(qw64, s.d_qw64, nwc * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        if (vw64) RC_CK(cudaMemcpyAsync(vw64, s.d_vw64, nwc * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        RC_CK(cudaStreamSynchronize(s.st));
        if (Q || sigma) scatter(s, Q, sigma);
        if (s.h_sc->status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values");
        return RC_OK;
    }

    // Fortran layout (0:imax+1, 0:jmax+1, 0:kloc+1) (mc_gpu_noint.cu:975-1005).
    void scatter(Slot<R> &s, float *Q, float *sigma) { scatter_from(s.h_Qc, s.h_Sc, s.h_Wq, s.h_Ws, Q, sigma); }

    // Float results of a batch member from the batch's packed host copy
    // (Q, sigma, wall flux, wall sigma one after the other at `pack`).
    int collect_packed(Slot<R> &s, const float *pack, float *Q, float *sigma) {
        std::string *err_ = &c->err;
        RC_FAILPOINT("collect");
        const size_t ncf = (size_t)c->p.imax * c->p.jmax * c->kloc;
        const size_t nwc = (size_t)2 * c->p.jmax * c->kloc;
        scatter_from(pack, pack + ncf, pack + 2 * ncf, pack + 2 * ncf + nwc, Q, sigma);
        if (s.h_sc->status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values");
        return RC_OK;
    }
    size_t packed_floats() const {
        return (size_t)2 * c->p.imax * c->p.jmax * c->kloc + (size_t)4 * c->p.jmax * c->kloc;
    }
    void pack_segments(Slot<R> &s, float *dst, CopySeg *seg) const {
        const long long ncf = (long long)c->p.imax * c->p.jmax * c->kloc;
        const long long nwc = 2LL * c->p.jmax * c->kloc;
        seg[0] = CopySeg{s.d_Qc, dst, ncf};
        seg[1] = CopySeg{s.d_Sc, dst + ncf, ncf};
        seg[2] = CopySeg{s.d_Wq, dst + 2 * ncf, nwc};
        seg[3] = CopySeg{s.d_Ws, dst + 2 * ncf + nwc, nwc};
    }

    void scatter_from(const float *Qc, const float *Sc, const float *Wq, const float *Ws, float *Q, float *sigma) {
        const rc_params &p = c->p;
        const int im = p.imax, jm = p.jmax, kl = c->kloc;
        const size_t sx = (size_t)im + 2, sy = (size_t)jm + 2;
        for (int k = 1; k <= kl; ++k)
            for (int j = 1; j <= jm; ++j) {
                const size_t src = ((size_t)(k - 1) * jm + (j - 1)) * im;
                const size_t dst = sx * ((size_t)j + sy * k);
                if (Q) memcpy(Q + dst + 1, Qc + src, im * sizeof(float));
                if (sigma) memcpy(sigma + dst + 1, Sc + src, im * sizeof(float));
                if (p.adiabw || p.adiabe) {
                    const size_t w = (size_t)(k - 1) * jm + (j - 1);
                    const size_t e = (size_t)jm * kl + w;
                    const bool cw = p.calcwalls && p.adiabw, ce = p.calcwalls && p.adiabe;
                    if (Q) {
                        Q[dst] = cw ? Wq[w] : 0.f;
                        Q[dst + im + 1] = ce ? Wq[e] : 0.f;
                    }
                    if (sigma) {
                        sigma[dst] = cw ? Ws[w] : 0.f;
                        sigma[dst + im + 1] = ce ? Ws[e] : 0.f;
                    }
                }
            }
    }

    int collect_device(rc_ticket t, double *q64, double *var64, double *qw64, double *vw64) {
        Range nv("rc_collect_device");
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown or already collected ticket");
        Slot<R> &s = *sp;
        const rc_params &p = c->p;
        const size_t ncf = (size_t)p.imax * p.jmax * c->kloc;
        const size_t nwc = (size_t)2 * p.jmax * c->kloc;
        if (q64) RC_CK(cudaMemcpyAsync(q64, s.d_q64, ncf * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
        if (var64) RC_CK(cudaMemcpyAsync(var64, s.d_var64, ncf * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
        if (qw64) RC_CK(cudaMemcpyAsync(qw64, s.d_qw64, nwc * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
        if (vw64) RC_CK(cudaMemcpyAsync(vw64, s.d_vw64, nwc * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
        RC_CK(cudaStreamSynchronize(s.st));
        s.state = 0;
        s.ticket = -1;
        if (s.h_sc->status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values");
        return RC_OK;
    }

    int device_results(rc_ticket t, const double **q64, const double **var64, const double **qw64,
                       const double **vw64) {
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown ticket");
        int rc = wait(*sp);
        if (rc) return rc;
        if (q64) *q64 = sp->d_q64;
        if (var64) *var64 = sp->d_var64;
        if (qw64) *qw64 = sp->d_qw64;
        if (vw64) *vw64 = sp->d_vw64;
        return RC_OK;
    }

    int info(rc_ticket t, rc_solve_info *out) {
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown ticket");
        int rc = wait(*sp);
        if (rc) return rc;
        const DScalars &d = *sp->h_sc;
        out->Tmax = __uint_as_float_host(d.tmax_bits);
        out->kappamax = (float)d.kappamax;
        out->Ibmax_fluid = (float)d.Ibmax_f;
        out->table_row = d.row;
        out->status = d.status | (d.bad_site << 8);
        out->bundles = (double)d.bundles;
        out->steps = (double)d.steps;
        float ms = 0.f;
        RC_CK(cudaEventElapsedTime(&ms, sp->e_march0, sp->e_march1));
        out->ms_device = ms;
        RC_CK(cudaEventElapsedTime(&ms, sp->e0, sp->e1));
        out->ms_solve = ms;
        return RC_OK;
    }

    static float __uint_as_float_host(unsigned int u) {
        float f;
        memcpy(&f, &u, 4);
        return f;
    }

    int trace(rc_ticket t, int n, const rc_bundle_id *ids, rc_trace_rec *out, int max_cells, int *cells) {
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown ticket");
        int rc = wait(*sp);
        if (rc) return rc;
        if (n <= 0) return RC_OK;
        rc_bundle_id *d_ids = nullptr;
        rc_trace_rec *d_out = nullptr;
        int *d_cells = nullptr;
        RC_CK(cudaMalloc((void **)&d_ids, n * sizeof(rc_bundle_id)));
        RC_CK(cudaMalloc((void **)&d_out, n * sizeof(rc_trace_rec)));
        if (cells && max_cells > 0) RC_CK(cudaMalloc((void **)&d_cells, (size_t)n * max_cells * 4 * sizeof(int)));
        RC_CK(cudaMemcpy(d_ids, ids, n * sizeof(rc_bundle_id), cudaMemcpyHostToDevice));
        if (d_cells) RC_CK(cudaMemset(d_cells, 0xff, (size_t)n * max_cells * 4 * sizeof(int)));
        if (nA > 0)
            k_trace<R, true><<<(n + 63) / 64, 64, 0, sp->st>>>(sp->d_desc, n, d_ids, d_out, d_cells ? max_cells : 0,
                                                               d_cells);
        else
            k_trace<R, false><<<(n + 63) / 64, 64, 0, sp->st>>>(sp->d_desc, n, d_ids, d_out, d_cells ? max_cells : 0,
                                                                d_cells);
        RC_CK(cudaGetLastError());
        RC_CK(cudaStreamSynchronize(sp->st));
        RC_CK(cudaMemcpy(out, d_out, n * sizeof(rc_trace_rec), cudaMemcpyDeviceToHost));
        if (d_cells)
            RC_CK(cudaMemcpy(cells, d_cells, (size_t)n * max_cells * 4 * sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(d_ids);
        cudaFree(d_out);
        if (d_cells) cudaFree(d_cells);
        return RC_OK;
    }

    int sample_bands(rc_ticket t, int kind, int n, const float *u_b, const float *u_g, int *nb, int *g) {
        std::string *err_ = &c->err;
        Slot<R> *sp = find_slot(t);
        if (!sp) return set_err(err_, RC_E_STATE, "unknown ticket");
        int rc = wait(*sp);
        if (rc) return rc;
        if (kind < 0 || kind > 2) return set_err(err_, RC_E_INVALID, "kind must be 0 (fluid), 1 or 2 (walls)");
        if (n <= 0) return RC_OK;
        float *d_u = nullptr;
        int *d_i = nullptr;
        RC_CK(cudaMalloc((void **)&d_u, 2 * (size_t)n * sizeof(float)));
        RC_CK(cudaMalloc((void **)&d_i, 2 * (size_t)n * sizeof(int)));
        RC_CK(cudaMemcpy(d_u, u_b, n * sizeof(float), cudaMemcpyHostToDevice));
        RC_CK(cudaMemcpy(d_u + n, u_g, n * sizeof(float), cudaMemcpyHostToDevice));
        k_sample_bands<R><<<(n + 127) / 128, 128, 0, sp->st>>>(sp->d_desc, kind, n, d_u, d_u + n, d_i, d_i + n);
        RC_CK(cudaGetLastError());
        RC_CK(cudaStreamSynchronize(sp->st));
        RC_CK(cudaMemcpy(nb, d_i, n * sizeof(int), cudaMemcpyDeviceToHost));
        RC_CK(cudaMemcpy(g, d_i + n, n * sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(d_u);
        cudaFree(d_i);
        return RC_OK;
    }
};

// dispatch helpers
template <typename F>
int with_impl(rc_ctx *c, F f) {
    if (c->dbl) return f(*static_cast<Impl<double> *>(c->impl));
    return f(*static_cast<Impl<float> *>(c->impl));
}

}  // namespace rc_detail
