// rc_solver.cu -- solver contexts, the per-solve pipeline on one stream,
// batched solves in one persistent launch (optionally a CUDA graph), bundle
// traces and the launch autotuner, behind the C ABI of radchan.h.
//
// Replaces the host side of the reference (mc_gpu_, get_results_,
// memory_copy_noint.cu): the grid, the tables and the Planck table are
// uploaded once per context and stay resident; a solve copies only the
// temperature field and runs
//   k_init_scalars -> k_tmax -> k_setup1 -> [k_grey_ib] -> k_setup2 ->
//   k_levels -> k_march -> k_tally
// on the context's stream without any host synchronisation.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "rc_host.h"
#include "rc_kernels.cuh"

using namespace rc;

namespace {
thread_local std::string g_err;

inline int set_err(std::string *dst, int code, const std::string &m) {
    if (dst) *dst = m;
    g_err = m;
    return code;
}
}  // namespace

#define RC_CK(call)                                                                                    \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return set_err(err_, RC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

// ---------------------------------------------------------------------------
// context implementation, templated on the march precision
// ---------------------------------------------------------------------------
namespace {
struct TallyOut {
    double *q64, *var64, *qw64, *vw64;
    float *Qc, *Sc, *Wq, *Ws;
};

template <typename R>
__global__ void k_tally_multi(const DSolve<R> *solves, const TallyOut *outs) {
    // one solve per blockIdx.y; reuse the single-solve body
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

struct SlotCommon {
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e_march0 = nullptr, e_march1 = nullptr;
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
    int state = 0;  // 0 free, 1 in flight, 2 finished (results pending)
    rc_ticket ticket = -1;
    int zstart = 1;
    int rpt = 0, block = 0;
    bool host_copied = false;
};

}  // namespace

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
    int num_sms = 148;
    bool has_tables = false;
    // precision-specific state
    void *impl = nullptr;  // Impl<float> or Impl<double>
    int dbl = 0;
};

namespace {

template <typename R>
struct Slot : SlotCommon {
    std::vector<uint16_t *> d_levT;
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
    std::vector<R *> d_xu, d_yu, d_zu;
    R *d_xc = nullptr, *d_yc = nullptr, *d_zc = nullptr;
    R *d_kt = nullptr, *d_Ibt = nullptr, *d_probg = nullptr, *d_prob = nullptr, *d_probq = nullptr;
    R *d_Ibw = nullptr, *d_Tnb = nullptr, *d_kP = nullptr, *d_wvl = nullptr, *d_wvr = nullptr, *d_wvc = nullptr;
    KIRow<R> *d_ki = nullptr;
    int nT = 0, nB = 0, nQ = 0;
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
            for (auto &p : s.d_levT) dfree(p);
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
            if (s.st) cudaStreamDestroy(s.st);
        }
        slots.clear();
        for (auto &p : d_xu) dfree(p);
        for (auto &p : d_yu) dfree(p);
        for (auto &p : d_zu) dfree(p);
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
        for (int l = 0; l < nl; ++l) {
            const GridLevel &g = c->grid[l];
            int rc = upload(d_xu[l], g.xu, err_);
            if (!rc) rc = upload(d_yu[l], g.yu, err_);
            if (!rc) rc = upload(d_zu[l], g.zu, err_);
            if (rc) return rc;
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
            LevelJobs &J = s.jobs;
            memset(&J, 0, sizeof(J));
            auto add_job = [&](void *dst, int type, int l, int face, long long n) {
                LevelJob &jb = J.job[J.njobs++];
                jb.dst = dst;
                jb.type = type;
                jb.nbi = (p.maxi[l] + 3) / 4;
                jb.nbj = (p.maxj[l] + 3) / 4;
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
                const long long nbr = (long long)((p.maxi[l] + 3) / 4) * ((p.maxj[l] + 3) / 4) * ((p.maxk[l] + 3) / 4);
                RC_CK(cudaMalloc((void **)&s.d_levT[l], nbr * 64 * sizeof(uint16_t)));
                RC_CK(cudaMemset(s.d_levT[l], 0, nbr * 64 * sizeof(uint16_t)));
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
        RC_CK(cudaFuncSetAttribute(k_march<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
        RC_CK(cudaFuncSetAttribute(k_march<R, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_opt_in));
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
        return RC_OK;
    }

    int set_tables(const TableSet &t) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        if (p.grey) return set_err(err_, RC_E_INVALID, "grey mode builds its own tables; rc_set_tables not used");
        if (t.nT != p.nT || t.nB != p.nB || t.nQ != p.nQ)
            return set_err(err_, RC_E_INVALID, "table dimensions differ from params nT/nB/nQ");
        if (t.nT < 2 || !(t.Tnb[1] > t.Tnb[0]))
            return set_err(err_, RC_E_INVALID, "table temperatures must be increasing");
        if (t.nT > 256) return set_err(err_, RC_E_INVALID, "at most 256 table temperatures");
        for (int i = 0; i < t.nT; ++i) {
            // the band search assumes non-decreasing cumulative probabilities
            for (int b = 1; b < t.nB; ++b)
                if (t.prob[(size_t)i * t.nB + b] < t.prob[(size_t)i * t.nB + b - 1])
                    return set_err(err_, RC_E_INVALID, "band cumulative probability decreases (prob_new2)");
            for (int b = 0; b < t.nB; ++b)
                for (int g = 1; g < t.nQ; ++g)
                    if (t.probg[((size_t)i * t.nB + b) * t.nQ + g] < t.probg[((size_t)i * t.nB + b) * t.nQ + g - 1])
                        return set_err(err_, RC_E_INVALID, "g cumulative probability decreases (prob_new2)");
        }
        for (int i = 2; i < t.nT; ++i) {
            // the lookups assume uniform spacing (pos = (T - T0)/dT)
            const double d0 = t.Tnb[1] - t.Tnb[0], di = t.Tnb[i] - t.Tnb[i - 1];
            if (fabs(di - d0) > 1e-3 * fabs(d0))
                return set_err(err_, RC_E_INVALID, "table temperatures must be uniformly spaced");
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
        return RC_OK;
    }

    // Work decomposition: items of rpt bundles, chunk count padded so that
    // the chunks of one (cell, replicate) never straddle a 32-item tile.
    void decompose(int rpt, int &nchunk, int &gsize, int &nparts) const {
        const int photmax = c->p.photmax;
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
            L.xu = d_xu[l];
            L.yu = d_yu[l];
            L.zu = d_zu[l];
            L.P = s.d_levT[l];
            L.nbi = (L.im + 3) / 4;
            L.nbj = (L.jm + 3) / 4;
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
        d.probq = d_probq;
        d.Ibw = d_Ibw;
        d.Pw0[0] = s.d_Tw0[0];
        d.Pw0[1] = s.d_Tw0[1];
        d.ki = p.grey ? s.d_ki_grey : d_ki;
        d.sc = s.d_sc;
        d.partial = s.d_partial;
        const long long ncf = (long long)p.imax * p.jmax * c->kloc;
        d.n_fluid_items = ncf * p.nVar * d.nchunk;
        d.n_items = d.n_fluid_items + (long long)d.nwalls * p.jmax * c->kloc * p.nVar * d.nchunk;
        d.n_tiles = (d.n_items + kWarp - 1) / kWarp;
        d.key0 = (uint32_t)p.seed;
        d.key1 = (uint32_t)(p.seed >> 32);
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

    // fdiv is exact when numerator * divisor < 2^64 at every division of the
    // item decomposition.
    bool decomposition_fits(const DSolve<R> &d) const {
        const long double lim = 18446744073709551615.0L;
        const long double n = (long double)d.n_items;
        return n * d.nchunk < lim && n * d.nVar < lim && n * c->p.imax < lim && n * c->p.jmax < lim &&
               n * (long double)d.nwc < lim;
    }

    size_t partial_count(int rpt) const {
        int nchunk, gsize, nparts;
        decompose(rpt, nchunk, gsize, nparts);
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

    size_t march_smem(int block, int rpt_max) const { return march_smem_bytes<R>(block, rpt_max); }

    static void (*march_fn(int minb))(MarchArgs) {
        return minb <= 2 ? k_march<R, 2> : minb == 3 ? k_march<R, 3> : k_march<R, 4>;
    }

    int launch_march(const DSolve<R> *d_solves, const long long *d_tiles, int nsolves, long long total_tiles,
                     unsigned long long *d_counter, int block, int rpt_max, cudaStream_t st, int minb = 0) {
        std::string *err_ = &c->err;
        if (minb <= 0) minb = c->minb;
        auto fn = march_fn(minb);
        const size_t smem = march_smem(block, rpt_max);
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

    // Everything up to the march on stream st: field copy, set-up kernels
    // and the descriptor (built into s.h_desc, copied to s.d_desc).
    int prepare(Slot<R> &s, const float *T_dev, int zstart, int rpt, cudaStream_t st) {
        std::string *err_ = &c->err;
        const rc_params &p = c->p;
        int rc = ensure_partial(s, rpt);
        if (rc) return rc;
        const size_t nfield = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
        if (T_dev) RC_CK(cudaMemcpyAsync(s.d_T, T_dev, nfield * sizeof(float), cudaMemcpyDeviceToDevice, st));
        else RC_CK(cudaMemcpyAsync(s.d_T, s.h_T, nfield * sizeof(float), cudaMemcpyHostToDevice, st));
        rc = enqueue_setup(s, st);
        if (rc) return rc;
        fill_desc(s, zstart, rpt, *s.h_desc);
        if (!decomposition_fits(*s.h_desc))
            return set_err(err_, RC_E_INVALID, "too many work items for one solve: raise rays_per_thread");
        RC_CK(cudaMemcpyAsync(s.d_desc, s.h_desc, sizeof(DSolve<R>), cudaMemcpyHostToDevice, st));
        k_patch_desc<R><<<1, 32, 0, st>>>(s.d_desc, s.d_sc);
        RC_CK(cudaGetLastError());
        TallyOut *o = s.h_out;
        o->q64 = s.d_q64;
        o->var64 = s.d_var64;
        o->qw64 = s.d_qw64;
        o->vw64 = s.d_vw64;
        o->Qc = s.d_Qc;
        o->Sc = s.d_Sc;
        o->Wq = s.d_Wq;
        o->Ws = s.d_Ws;
        RC_CK(cudaMemcpyAsync(s.d_out, s.h_out, sizeof(TallyOut), cudaMemcpyHostToDevice, st));
        s.zstart = zstart;
        s.rpt = rpt;
        return RC_OK;
    }

    int launch_tally(const DSolve<R> *d_solves, const TallyOut *d_outs, int nsolves, long long max_cells,
                     cudaStream_t st) {
        std::string *err_ = &c->err;
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
        RC_CK(cudaEventRecord(s.e_march0, s.st));
        rc = launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, c->block, rpt, s.st);
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
    // decomposition and the FP64 summation grouping.
    int autotune(const float *T, int zstart, int pilot, int *rpt_out, int *block_out, int *occ_out) {
        std::string *err_ = &c->err;
        int rc = check_solve_args(T, zstart);
        if (rc) return rc;
        Slot<R> *sp = free_slot();
        if (!sp) return set_err(err_, RC_E_BUSY, "all solve slots in use");
        Slot<R> &s = *sp;
        const int saved_photmax = c->p.photmax;
        if (pilot > 0) c->p.photmax = pilot;
        rc = stage_host_field(s, T);
        float best = 3.4e38f;
        int brpt = c->rpt, bblock = c->block, bminb = c->minb;
        const int rpts[] = {2, 4, 8, 16, 32};
        const int blocks[] = {128, 256};
        const int minbs[] = {2, 3, 4};
        for (int oi = 0; oi < 3 && !rc; ++oi)
        for (int bi = 0; bi < 2 && !rc; ++bi)
            for (int ri = 0; ri < 5 && !rc; ++ri) {
                const int rpt = rpts[ri], block = blocks[bi], minb = minbs[oi];
                if (march_smem(block, rpt) > (size_t)smem_opt_in) continue;
                float tot = 0.f;
                for (int rep = 0; rep < 2 && !rc; ++rep) {
                    rc = prepare(s, nullptr, zstart, rpt, s.st);
                    if (rc) break;
                    s.h_tiles[0] = 0;
                    s.h_tiles[1] = s.h_desc->n_tiles;
                    cudaError_t e = cudaMemcpyAsync(s.d_tiles, s.h_tiles, 2 * sizeof(long long),
                                                    cudaMemcpyHostToDevice, s.st);
                    if (e != cudaSuccess) {
                        rc = set_err(err_, RC_E_CUDA, cudaGetErrorString(e));
                        break;
                    }
                    cudaEventRecord(s.e_march0, s.st);
                    rc = launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, block, rpt, s.st, minb);
                    if (rc) break;
                    cudaEventRecord(s.e_march1, s.st);
                    e = cudaEventSynchronize(s.e_march1);
                    if (e != cudaSuccess) {
                        rc = set_err(err_, RC_E_CUDA, cudaGetErrorString(e));
                        break;
                    }
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, s.e_march0, s.e_march1);
                    if (rep > 0) tot += ms;  // first run warms up
                }
                if (!rc && tot < best) {
                    best = tot;
                    brpt = rpt;
                    bblock = block;
                    bminb = minb;
                }
            }
        c->p.photmax = saved_photmax;
        if (rc) return rc;
        c->rpt = brpt;
        c->block = bblock;
        c->minb = bminb;
        if (rpt_out) *rpt_out = brpt;
        if (block_out) *block_out = bblock;
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
    void scatter(Slot<R> &s, float *Q, float *sigma) {
        const rc_params &p = c->p;
        const int im = p.imax, jm = p.jmax, kl = c->kloc;
        const size_t sx = (size_t)im + 2, sy = (size_t)jm + 2;
        for (int k = 1; k <= kl; ++k)
            for (int j = 1; j <= jm; ++j) {
                const size_t src = ((size_t)(k - 1) * jm + (j - 1)) * im;
                const size_t dst = sx * ((size_t)j + sy * k);
                if (Q) memcpy(Q + dst + 1, s.h_Qc + src, im * sizeof(float));
                if (sigma) memcpy(sigma + dst + 1, s.h_Sc + src, im * sizeof(float));
                if (p.adiabw || p.adiabe) {
                    const size_t w = (size_t)(k - 1) * jm + (j - 1);
                    const size_t e = (size_t)jm * kl + w;
                    const bool cw = p.calcwalls && p.adiabw, ce = p.calcwalls && p.adiabe;
                    if (Q) {
                        Q[dst] = cw ? s.h_Wq[w] : 0.f;
                        Q[dst + im + 1] = ce ? s.h_Wq[e] : 0.f;
                    }
                    if (sigma) {
                        sigma[dst] = cw ? s.h_Ws[w] : 0.f;
                        sigma[dst + im + 1] = ce ? s.h_Ws[e] : 0.f;
                    }
                }
            }
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
        out->status = d.status;
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
        k_trace<R><<<(n + 63) / 64, 64, 0, sp->st>>>(sp->d_desc, n, d_ids, d_out, d_cells ? max_cells : 0, d_cells);
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
};

// dispatch helpers
template <typename F>
int with_impl(rc_ctx *c, F f) {
    if (c->dbl) return f(*static_cast<Impl<double> *>(c->impl));
    return f(*static_cast<Impl<float> *>(c->impl));
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI: parameters, tables, geometry
// ---------------------------------------------------------------------------
extern "C" {

int rc_params_default(rc_params *p) {
    if (!p) return set_err(nullptr, RC_E_INVALID, "NULL params");
    return params_default(*p);
}

int rc_params_from_headers(const char *param_h, const char *narrowband_h, rc_params *p) {
    if (!param_h || !p) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::string err;
    int rc = params_from_headers(param_h, narrowband_h ? narrowband_h : "", *p, err);
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_params_validate(const rc_params *p, char *msg, size_t msglen) {
    if (!p) return set_err(nullptr, RC_E_INVALID, "NULL params");
    std::string err;
    int rc = params_validate(*p, err);
    if (msg && msglen) {
        snprintf(msg, msglen, "%s", err.c_str());
    }
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_tables_synthetic(const rc_synth_spec *spec, rc_table_set **out) {
    if (!spec || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    auto *ts = new rc_table_set();
    std::string err;
    int rc = tables_synthetic(*spec, ts->ts, err);
    if (rc) {
        delete ts;
        return set_err(nullptr, rc, err);
    }
    *out = ts;
    return RC_OK;
}

int rc_tables_read_dir(const char *dir, int nT, int nB, int nQ, rc_table_set **out) {
    if (!dir || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    auto *ts = new rc_table_set();
    std::string err;
    int rc = tables_read_dir(dir, nT, nB, nQ, ts->ts, err);
    if (rc) {
        delete ts;
        return set_err(nullptr, rc, err);
    }
    *out = ts;
    return RC_OK;
}

int rc_tables_write_dir(const rc_table_set *ts, const char *dir) {
    if (!ts || !dir) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::string err;
    int rc = tables_write_dir(ts->ts, dir, err);
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_tables_view(const rc_table_set *ts, rc_tables *view) {
    if (!ts || !view) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    ts->ts.view(view);
    return RC_OK;
}

void rc_tables_free(rc_table_set *ts) { delete ts; }

int rc_grid_level(const rc_params *p, int level, float *xu, float *yu, float *zu, float *x, float *y, float *z) {
    if (!p) return set_err(nullptr, RC_E_INVALID, "NULL params");
    std::string err;
    if (params_validate(*p, err)) return set_err(nullptr, RC_E_INVALID, err);
    if (level < 0 || level >= p->grid_num) return set_err(nullptr, RC_E_INVALID, "level out of range");
    GridLevel g;
    build_grid_level(*p, level, g);
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

// ---------------------------------------------------------------------------
// C ABI: contexts
// ---------------------------------------------------------------------------
int rc_create(const rc_params *p, int device, rc_ctx **out) {
    if (!p || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::string err;
    if (params_validate(*p, err)) return set_err(nullptr, RC_E_INVALID, err);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_err(nullptr, RC_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return set_err(nullptr, RC_E_INVALID, "device index out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_err(nullptr, RC_E_CUDA, cudaGetErrorString(e));
    auto *c = new rc_ctx();
    c->p = *p;
    c->device = device;
    c->kloc = p->kmax / p->p_col;
    wall_types(*p, c->wt);
    c->grid.resize(p->grid_num);
    for (int l = 0; l < p->grid_num; ++l) build_grid_level(*p, l, c->grid[l]);
    c->dbl = p->floatpoint == 1;
    // measured best on B200 for the 64^3 narrow-band and 32^3 grey channels:
    // 4 bundles per work item, 256-thread blocks, 64-register budget (FP32);
    // the FP64 ray state needs the larger register budget
    c->rpt = 4;
    c->block = 256;
    c->minb = c->dbl ? 2 : 4;
    int rc;
    if (c->dbl) {
        auto *im = new Impl<double>();
        im->c = c;
        c->impl = im;
        rc = im->init(2);
    } else {
        auto *im = new Impl<float>();
        im->c = c;
        c->impl = im;
        rc = im->init(2);
    }
    if (rc) {
        std::string m = c->err;
        rc_destroy(c);
        return set_err(nullptr, rc, m);
    }
    *out = c;
    return RC_OK;
}

int rc_set_tables(rc_ctx *c, const rc_tables *t) {
    if (!c || !t) return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    TableSet ts;
    ts.from_view(t);
    return with_impl(c, [&](auto &im) { return im.set_tables(ts); });
}

int rc_solve_async(rc_ctx *c, const float *T, int zstart, rc_ticket *ticket) {
    if (!c || !ticket) return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.solve(T, false, zstart, ticket); });
}

int rc_solve_device_async(rc_ctx *c, const float *T_dev, int zstart, rc_ticket *ticket) {
    if (!c || !ticket) return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.solve(T_dev, true, zstart, ticket); });
}

int rc_collect(rc_ctx *c, rc_ticket t, float *Q, float *sigma, double *q64, double *var64, double *qw64,
               double *vw64) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.collect(t, Q, sigma, q64, var64, qw64, vw64); });
}

int rc_device_results(rc_ctx *c, rc_ticket t, const double **q64, const double **var64, const double **qw64,
                      const double **vw64) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.device_results(t, q64, var64, qw64, vw64); });
}

int rc_solve_info_get(rc_ctx *c, rc_ticket t, rc_solve_info *info) {
    if (!c || !info) return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.info(t, info); });
}

int rc_set_launch(rc_ctx *c, int rays_per_thread, int block_threads, int sort_bands, int occupancy) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    if (rays_per_thread > 0) {
        if (rays_per_thread > 64 || (rays_per_thread & (rays_per_thread - 1)))
            return set_err(&c->err, RC_E_INVALID, "rays_per_thread must be a power of two <= 64");
        c->rpt = rays_per_thread;
    }
    if (block_threads > 0) {
        if (block_threads != 128 && block_threads != 256)
            return set_err(&c->err, RC_E_INVALID, "block_threads must be 128 or 256");
        c->block = block_threads;
    }
    if (sort_bands >= 0) c->sort = sort_bands;
    if (occupancy > 0) {
        if (occupancy < 2 || occupancy > 4) return set_err(&c->err, RC_E_INVALID, "occupancy must be 2, 3 or 4");
        c->minb = occupancy;
    }
    return RC_OK;
}

int rc_get_launch(rc_ctx *c, int *rays_per_thread, int *block_threads, int *sort_bands, int *occupancy) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    if (rays_per_thread) *rays_per_thread = c->rpt;
    if (block_threads) *block_threads = c->block;
    if (sort_bands) *sort_bands = c->sort;
    if (occupancy) *occupancy = c->minb;
    return RC_OK;
}

int rc_trace(rc_ctx *c, rc_ticket t, int n, const rc_bundle_id *ids, rc_trace_rec *out, int max_cells, int *cells) {
    if (!c || (n > 0 && (!ids || !out))) return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.trace(t, n, ids, out, max_cells, cells); });
}

int rc_destroy(rc_ctx *c) {
    if (!c) return RC_OK;
    cudaSetDevice(c->device);
    if (c->impl) {
        if (c->dbl) delete static_cast<Impl<double> *>(c->impl);
        else delete static_cast<Impl<float> *>(c->impl);
    }
    delete c;
    return RC_OK;
}

int rc_last_error(const rc_ctx *c, char *buf, size_t len) {
    const std::string &m = c ? c->err : g_err;
    if (buf && len) snprintf(buf, len, "%s", m.c_str());
    return RC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batched solves: many contexts' solves in one persistent launch
// ---------------------------------------------------------------------------
struct rc_batch {
    int device = 0;
    int use_graph = 1;
    int dbl = -1;
    struct Member {
        rc_ctx *ctx;
        void *slot;
        int zstart;
    };
    std::vector<Member> m;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool built = false;
    void *d_solves = nullptr, *h_solves = nullptr;
    long long *d_tiles = nullptr, *h_tiles = nullptr;
    TallyOut *d_outs = nullptr, *h_outs = nullptr;
    unsigned long long *d_counter = nullptr;
    size_t cap = 0;
    std::string err;
};

namespace {

template <typename R>
int batch_reserve(rc_batch *b, size_t n) {
    std::string *err_ = &b->err;
    if (n <= b->cap) return RC_OK;
    if (b->d_solves) cudaFree(b->d_solves);
    if (b->h_solves) cudaFreeHost(b->h_solves);
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->h_tiles) cudaFreeHost(b->h_tiles);
    if (b->d_outs) cudaFree(b->d_outs);
    if (b->h_outs) cudaFreeHost(b->h_outs);
    RC_CK(cudaMalloc(&b->d_solves, n * sizeof(DSolve<R>)));
    RC_CK(cudaHostAlloc(&b->h_solves, n * sizeof(DSolve<R>), cudaHostAllocDefault));
    RC_CK(cudaMalloc((void **)&b->d_tiles, (n + 1) * sizeof(long long)));
    RC_CK(cudaHostAlloc((void **)&b->h_tiles, (n + 1) * sizeof(long long), cudaHostAllocDefault));
    RC_CK(cudaMalloc((void **)&b->d_outs, n * sizeof(TallyOut)));
    RC_CK(cudaHostAlloc((void **)&b->h_outs, n * sizeof(TallyOut), cudaHostAllocDefault));
    b->cap = n;
    return RC_OK;
}

// The whole batch on b->st: per member field copy + set-up, one march
// over every member's tiles, one tally launch, scalars back.
template <typename R>
int batch_enqueue(rc_batch *b) {
    std::string *err_ = &b->err;
    const size_t n = b->m.size();
    int rc = batch_reserve<R>(b, n);
    if (rc) return rc;
    DSolve<R> *hs = static_cast<DSolve<R> *>(b->h_solves);
    int rpt_max = 1, block = 256;
    long long max_cells = 1;
    b->h_tiles[0] = 0;
    for (size_t i = 0; i < n; ++i) {
        rc_ctx *c = b->m[i].ctx;
        Impl<R> &im = *static_cast<Impl<R> *>(c->impl);
        Slot<R> &s = *static_cast<Slot<R> *>(b->m[i].slot);
        rc = im.prepare(s, nullptr, b->m[i].zstart, c->rpt, b->st);
        if (rc) return set_err(err_, rc, c->err);
        hs[i] = *s.h_desc;
        b->h_outs[i] = *s.h_out;
        b->h_tiles[i + 1] = b->h_tiles[i] + s.h_desc->n_tiles;
        rpt_max = std::max(rpt_max, c->rpt);
        if (i == 0) block = c->block;
        max_cells = std::max(max_cells, im.tally_cells());
    }
    // descriptors with their run-time fields already patched on the device
    for (size_t i = 0; i < n; ++i) {
        Slot<R> &s = *static_cast<Slot<R> *>(b->m[i].slot);
        RC_CK(cudaMemcpyAsync(static_cast<DSolve<R> *>(b->d_solves) + i, s.d_desc, sizeof(DSolve<R>),
                              cudaMemcpyDeviceToDevice, b->st));
    }
    RC_CK(cudaMemcpyAsync(b->d_tiles, b->h_tiles, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, b->st));
    RC_CK(cudaMemcpyAsync(b->d_outs, b->h_outs, n * sizeof(TallyOut), cudaMemcpyHostToDevice, b->st));
    Impl<R> &im0 = *static_cast<Impl<R> *>(b->m[0].ctx->impl);
    rc = im0.launch_march(static_cast<const DSolve<R> *>(b->d_solves), b->d_tiles, (int)n, b->h_tiles[n],
                          b->d_counter, block, rpt_max, b->st);
    if (rc) return set_err(err_, rc, b->m[0].ctx->err);
    rc = im0.launch_tally(static_cast<const DSolve<R> *>(b->d_solves), b->d_outs, (int)n, max_cells, b->st);
    if (rc) return set_err(err_, rc, b->m[0].ctx->err);
    for (size_t i = 0; i < n; ++i) {
        Slot<R> &s = *static_cast<Slot<R> *>(b->m[i].slot);
        RC_CK(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(DScalars), cudaMemcpyDeviceToHost, b->st));
    }
    return RC_OK;
}

template <typename R>
int batch_ensure_scratch(rc_batch *b) {
    for (auto &mm : b->m) {
        Impl<R> &im = *static_cast<Impl<R> *>(mm.ctx->impl);
        Slot<R> &s = *static_cast<Slot<R> *>(mm.slot);
        int rc = im.ensure_partial(s, mm.ctx->rpt);
        if (rc) return set_err(&b->err, rc, mm.ctx->err);
    }
    return RC_OK;
}

template <typename R>
void batch_release(rc_batch *b) {
    for (auto &mm : b->m) {
        Slot<R> &s = *static_cast<Slot<R> *>(mm.slot);
        s.state = 0;
        s.ticket = -1;
    }
}

}  // namespace

extern "C" {

int rc_autotune(rc_ctx *c, const float *T, int zstart, int pilot_photmax, int *rays_per_thread, int *block_threads,
                int *sort_bands) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) {
        return im.autotune(T, zstart, pilot_photmax, rays_per_thread, block_threads, sort_bands);
    });
}

int rc_batch_create(int device, int use_graph, rc_batch **out) {
    if (!out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_err(nullptr, RC_E_CUDA, cudaGetErrorString(e));
    auto *b = new rc_batch();
    b->device = device;
    b->use_graph = use_graph ? 1 : 0;
    std::string *err_ = &b->err;
    auto fail = [&](cudaError_t ee) {
        std::string m = cudaGetErrorString(ee);
        rc_batch_destroy(b);
        return set_err(nullptr, RC_E_CUDA, m);
    };
    if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&b->e0)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&b->e1)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void **)&b->d_counter, sizeof(unsigned long long))) != cudaSuccess) return fail(e);
    (void)err_;
    *out = b;
    return RC_OK;
}

int rc_batch_add(rc_batch *b, rc_ctx *c, const float *T_host, int zstart) {
    if (!b || !c || !T_host) return set_err(b ? &b->err : nullptr, RC_E_INVALID, "NULL argument");
    if (c->device != b->device) return set_err(&b->err, RC_E_INVALID, "context on another device");
    if (b->dbl >= 0 && b->dbl != c->dbl) return set_err(&b->err, RC_E_INVALID, "mixed precision in one batch");
    cudaSetDevice(c->device);
    int rc = with_impl(c, [&](auto &im) {
        int r = im.check_solve_args(T_host, zstart);
        if (r) return r;
        auto *s = im.free_slot();
        if (!s) return set_err(&c->err, RC_E_BUSY, "no free slot in context");
        r = im.stage_host_field(*s, T_host);
        if (r) return r;
        s->state = 3;  // reserved by the batch
        rc_batch::Member mm;
        mm.ctx = c;
        mm.slot = s;
        mm.zstart = zstart;
        b->m.push_back(mm);
        return RC_OK;
    });
    if (rc) return set_err(&b->err, rc, c->err);
    b->dbl = c->dbl;
    b->built = false;
    return RC_OK;
}

int rc_batch_run(rc_batch *b) {
    if (!b) return set_err(nullptr, RC_E_INVALID, "NULL batch");
    if (b->m.empty()) return set_err(&b->err, RC_E_STATE, "empty batch");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    int rc = b->dbl ? batch_ensure_scratch<double>(b) : batch_ensure_scratch<float>(b);
    if (rc) return rc;
    // all allocations happen before any stream capture
    rc = b->dbl ? batch_reserve<double>(b, b->m.size()) : batch_reserve<float>(b, b->m.size());
    if (rc) return rc;
    if (!b->use_graph) {
        RC_CK(cudaEventRecord(b->e0, b->st));
        rc = b->dbl ? batch_enqueue<double>(b) : batch_enqueue<float>(b);
        if (rc) return rc;
        RC_CK(cudaEventRecord(b->e1, b->st));
        return RC_OK;
    }
    if (!b->built) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        if (b->graph) {
            cudaGraphDestroy(b->graph);
            b->graph = nullptr;
        }
        RC_CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        rc = b->dbl ? batch_enqueue<double>(b) : batch_enqueue<float>(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->st, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return set_err(err_, RC_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        b->graph = g;
        RC_CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->built = true;
    }
    RC_CK(cudaEventRecord(b->e0, b->st));
    RC_CK(cudaGraphLaunch(b->exec, b->st));
    RC_CK(cudaEventRecord(b->e1, b->st));
    return RC_OK;
}

int rc_batch_wait(rc_batch *b, float *ms_device) {
    if (!b) return set_err(nullptr, RC_E_INVALID, "NULL batch");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    RC_CK(cudaEventSynchronize(b->e1));
    if (ms_device) RC_CK(cudaEventElapsedTime(ms_device, b->e0, b->e1));
    return RC_OK;
}

int rc_batch_collect(rc_batch *b, int index, float *Q, float *sigma, double *q64, double *var64, double *qw64,
                     double *vw64) {
    if (!b || index < 0 || index >= (int)b->m.size())
        return set_err(b ? &b->err : nullptr, RC_E_INVALID, "bad batch index");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    RC_CK(cudaEventSynchronize(b->e1));
    rc_ctx *c = b->m[index].ctx;
    void *slot = b->m[index].slot;
    int rc;
    if (c->dbl)
        rc = static_cast<Impl<double> *>(c->impl)->copy_out(*static_cast<Slot<double> *>(slot), Q, sigma, q64, var64,
                                                             qw64, vw64);
    else
        rc = static_cast<Impl<float> *>(c->impl)->copy_out(*static_cast<Slot<float> *>(slot), Q, sigma, q64, var64,
                                                           qw64, vw64);
    if (rc) return set_err(&b->err, rc, c->err);
    return RC_OK;
}

int rc_batch_destroy(rc_batch *b) {
    if (!b) return RC_OK;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->dbl == 1) batch_release<double>(b);
    else if (b->dbl == 0) batch_release<float>(b);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_solves) cudaFree(b->d_solves);
    if (b->h_solves) cudaFreeHost(b->h_solves);
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->h_tiles) cudaFreeHost(b->h_tiles);
    if (b->d_outs) cudaFree(b->d_outs);
    if (b->h_outs) cudaFreeHost(b->h_outs);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return RC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solve into caller-provided device arrays with library-owned scratch, for
// callers that must not allocate device memory while they run.
// ---------------------------------------------------------------------------
namespace {

// Partial sums of the march (one double per (cell, replicate, part)) live in
// this file-scope device array instead of a cudaMalloc'd buffer.  Every GPU
// that loads the library holds it until the process exits.
constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;  // 64 MiB
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[128] = {};

// Device address of the scratch array on `device` (which must be current).
// In host code g_noalloc_scratch is only a host-side stand-in for the symbol,
// so the address is looked up once per device and cached.
int noalloc_scratch(int device, double **out, std::string *err_) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (device < 0 || device >= 128) return set_err(err_, RC_E_INVALID, "device index out of range");
    if (!g_noalloc_ptr[device]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_err(err_, RC_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return RC_OK;
}

template <typename R>
int solve_noalloc_t(rc_ctx *c, const float *T_dev, int zstart, double *q64, double *var64, double *qw64,
                    double *vw64) {
    Impl<R> &im = *static_cast<Impl<R> *>(c->impl);
    std::string *err_ = &c->err;
    const rc_params &p = c->p;
    int rc = im.check_solve_args(T_dev, zstart);
    if (rc) return rc;
    if (!q64 || !var64) return set_err(err_, RC_E_INVALID, "q64 and var64 output arrays are required");
    const int rpt = c->rpt;
    const size_t need = im.partial_count(rpt);
    if (need > kNoAllocScratchDoubles)
        return set_err(err_, RC_E_INVALID,
                       "rc_solve_noalloc: this solve needs " + std::to_string(need) +
                           " doubles of scratch but the static array holds " +
                           std::to_string(kNoAllocScratchDoubles) +
                           " (64 MiB); raise rays_per_thread or use rc_solve_device_async");
    double *scratch = nullptr;
    rc = noalloc_scratch(c->device, &scratch, err_);
    if (rc) return rc;
    Slot<R> *sp = im.free_slot();
    if (!sp) return set_err(err_, RC_E_BUSY, "all solve slots in use: collect a ticket first");
    Slot<R> &s = *sp;
    cudaStream_t st = s.st;
    const size_t nfield = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
    RC_CK(cudaMemcpyAsync(s.d_T, T_dev, nfield * sizeof(float), cudaMemcpyDeviceToDevice, st));
    rc = im.enqueue_setup(s, st);
    if (rc) return rc;
    im.fill_desc(s, zstart, rpt, *s.h_desc);
    s.h_desc->partial = scratch;
    if (!im.decomposition_fits(*s.h_desc))
        return set_err(err_, RC_E_INVALID, "too many work items for one solve: raise rays_per_thread");
    RC_CK(cudaMemcpyAsync(s.d_desc, s.h_desc, sizeof(DSolve<R>), cudaMemcpyHostToDevice, st));
    k_patch_desc<R><<<1, 32, 0, st>>>(s.d_desc, s.d_sc);
    RC_CK(cudaGetLastError());
    TallyOut *o = s.h_out;
    o->q64 = q64;
    o->var64 = var64;
    o->qw64 = qw64;
    o->vw64 = vw64;
    o->Qc = s.d_Qc;
    o->Sc = s.d_Sc;
    o->Wq = s.d_Wq;
    o->Ws = s.d_Ws;
    RC_CK(cudaMemcpyAsync(s.d_out, s.h_out, sizeof(TallyOut), cudaMemcpyHostToDevice, st));
    s.h_tiles[0] = 0;
    s.h_tiles[1] = s.h_desc->n_tiles;
    RC_CK(cudaMemcpyAsync(s.d_tiles, s.h_tiles, 2 * sizeof(long long), cudaMemcpyHostToDevice, st));
    rc = im.launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, c->block, rpt, st);
    if (rc) return rc;
    rc = im.launch_tally(s.d_desc, s.d_out, 1, im.tally_cells(), st);
    if (rc) return rc;
    RC_CK(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(DScalars), cudaMemcpyDeviceToHost, st));
    RC_CK(cudaStreamSynchronize(st));
    if (s.h_sc->status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values");
    return RC_OK;
}

}  // namespace

extern "C" int rc_solve_noalloc(rc_ctx *c, const float *T_dev, int zstart, double *q64_dev, double *var64_dev,
                                double *qw64_dev, double *vw64_dev) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return set_err(&c->err, RC_E_CUDA, cudaGetErrorString(e));
    if (c->dbl) return solve_noalloc_t<double>(c, T_dev, zstart, q64_dev, var64_dev, qw64_dev, vw64_dev);
    return solve_noalloc_t<float>(c, T_dev, zstart, q64_dev, var64_dev, qw64_dev, vw64_dev);
}
