// rc_dns.cu -- the channel DNS's use of a finished solve, fused into one
// kernel over the solve's device results (rc_dns_source*, radchan.h).
//
// The reference runs, after every radStep-th DNS step (src/dns/channel.f:
// 249-266): GET_RESULTS (device -> host Q, sigma as float), fix_rad
// (fixvar.f:179-242: MPI_Allreduce over the k communicator, then per cell of
// the rank's j pencil Qnew = Q/stefan/Tin^4, walls also /Height,
// Varnew = sigma/stefan/Tin^4), fix_kappa (fixvar.f:16-43: Knew = kP at
// T1 Tin by linear_int), and the loop Qnew *= underrelax,
// Gnew = 4 T1^4 - Qnew/Knew.  Here one launch reads the float results that
// get_results_ would return straight from HBM and writes the four double
// arrays; with one solver per pencil the allreduce is the identity (each
// cell has exactly one contributing GPU), so it has no counterpart.
//
// Arithmetic follows the Fortran statement by statement in double
// precision, without contraction (-fmad=false): two roundings for
// Q/stefan/Tin^4, the slope of linear_int as (y(t+1)-y(t))/(x(t+1)-x(t))
// (computed once per table row on the host, the same IEEE operation), then
// slope*(x0-x(t)) + y(t).  Tin^4 is pow(Tin, 4.0) on the host, as Tin**4.
// is in the DNS.  T1**4. is evaluated as (T1 T1)(T1 T1).
#include <cmath>
#include <thread>
#include <vector>

#include "rc_impl.cuh"

using namespace rc_detail;

namespace {

struct DnsArgs {
    const float *Qc, *Sc, *Wq, *Ws;  // solve results: [kloc][jmax][imax], walls [2][kloc][jmax]
    const double *T1;                // (0:imax+1, 0:jn+1, 0:kloc+1)
    double *Qnew, *Varnew, *Knew, *Gnew;  // (0:imax+1, jn, kloc)
    unsigned long long *n_clamped;
    double stefan, Tin, Tin4, Height, underrelax;
    int imax, jmax, kloc, jstart, jn, west, east;
    int nT, dT;
    unsigned long long Mnx, Mjn, MdT;  // fdiv multipliers of imax+2, jn, dT
    double Tnb[RC_DNS_MAX_T], kP[RC_DNS_MAX_T], slope[RC_DNS_MAX_T];
};

// One thread per output cell (grid-stride), i fastest, so every load and
// store of a warp is contiguous; (i, j, k) and linear_int's row come from
// exact multiply-high divisions (fdiv) instead of integer division.  The
// kernel is bound by instruction issue: the five IEEE double divisions the
// Fortran's statement order requires take most of its ~245 instructions per
// cell (measured on B200; 6 resident blocks per SM were 2-3% faster than 4,
// two cells per thread no faster).
__global__ void __launch_bounds__(256, 6) k_dns_source(const __grid_constant__ DnsArgs a) {
    __shared__ double sT[RC_DNS_MAX_T], sK[RC_DNS_MAX_T], sS[RC_DNS_MAX_T];
    for (int t = threadIdx.x; t < a.nT; t += blockDim.x) {
        sT[t] = a.Tnb[t];
        sK[t] = a.kP[t];
        sS[t] = a.slope[t];
    }
    __syncthreads();
    const int nx = a.imax + 2;
    const unsigned long long n = (unsigned long long)nx * a.jn * a.kloc;
    unsigned int clamped = 0;
    for (unsigned long long c = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; c < n;
         c += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long r = fdiv(c, a.Mnx);  // (j, k) row
        const int i = (int)(c - r * nx);
        const unsigned long long k0 = fdiv(r, a.Mjn);
        const int jl = (int)(r - k0 * a.jn) + 1;  // 1..jn, local to the pencil
        const int kl = (int)k0 + 1;               // 1..kloc
        const int jg = a.jstart + jl - 1;         // 1..jmax, the solve's j
        const long long wcell = (long long)(kl - 1) * a.jmax + (jg - 1);
        const bool wall = (i == 0) || (i == nx - 1);
        float q = 0.f, s = 0.f;
        if (wall) {
            // get_results_ writes 0 on a wall whose flux is not computed
            if (i == 0 ? a.west : a.east) {
                const long long w = (i == 0 ? 0LL : (long long)a.jmax * a.kloc) + wcell;
                q = __ldg(a.Wq + w);
                s = __ldg(a.Ws + w);
            }
        } else {
            q = __ldg(a.Qc + (wcell * a.imax + (i - 1)));
            s = __ldg(a.Sc + (wcell * a.imax + (i - 1)));
        }
        const double T1 = __ldg(a.T1 + (i + (long long)nx * (jl + (long long)(a.jn + 2) * kl)));
        double Qn = (double)q / a.stefan / a.Tin4;
        if (wall) Qn = Qn / a.Height;
        const double Vn = (double)s / a.stefan / a.Tin4;
        const double x0 = T1 * a.Tin;
        const double d = x0 - sT[0];
        // t = int(x0 - x(1)) / int(x(2) - x(1)): both truncate toward zero
        int t;
        if (d > -2147483648.0 && d < 2147483648.0) {
            const int ti = (int)d;
            const int tq = (int)fdiv((unsigned long long)(ti < 0 ? -(long long)ti : ti), a.MdT);
            t = ti < 0 ? -tq : tq;
        } else {
            t = (d > 0.0) ? a.nT : -1;  // far out of range, or NaN
        }
        if (t < 0 || t > a.nT - 2) {
            ++clamped;
            t = (t < 0) ? 0 : a.nT - 2;
        }
        const double K = sS[t] * (x0 - sT[t]) + sK[t];
        Qn = Qn * a.underrelax;
        const double t2 = T1 * T1;
        const double G = 4.0 * (t2 * t2) - Qn / K;
        a.Qnew[c] = Qn;
        a.Varnew[c] = Vn;
        a.Knew[c] = K;
        a.Gnew[c] = G;
    }
    if (a.n_clamped) {
        const unsigned int w = __reduce_add_sync(0xffffffffu, clamped);
        if ((threadIdx.x & 31) == 0 && w) atomicAdd(a.n_clamped, (unsigned long long)w);
    }
}

// Validate the coupling against the context and fill the kernel arguments
// except the array pointers.
int dns_args(const rc_ctx *c, const rc_dns_coupling *cfg, DnsArgs &a, std::string *err_) {
    if (!cfg) return set_err(err_, RC_E_INVALID, "NULL coupling");
    const rc_params &p = c->p;
    if (!cfg->Tnb || !cfg->kP) return set_err(err_, RC_E_INVALID, "coupling Tnb/kP is NULL");
    if (cfg->nTemp < 2 || cfg->nTemp > RC_DNS_MAX_T)
        return set_err(err_, RC_E_INVALID, "coupling nTemp must be in 2..RC_DNS_MAX_T");
    if (cfg->jstart < 1 || cfg->jend > p.jmax || cfg->jstart > cfg->jend)
        return set_err(err_, RC_E_INVALID, "coupling j range outside 1..jmax");
    // fdiv(c, M) is exact when c * divisor < 2^64: c < cells, divisor <= imax+2
    if ((long double)(p.imax + 2) * (cfg->jend - cfg->jstart + 1) * c->kloc * (p.imax + 2) >= 1.8e19L)
        return set_err(err_, RC_E_INVALID, "coupling pencil too large");
    if (!(cfg->Tin > 0.0) || !std::isfinite(cfg->Tin) || cfg->stefan == 0.0 || cfg->Height == 0.0)
        return set_err(err_, RC_E_INVALID, "coupling needs Tin > 0 and non-zero stefan and Height");
    const double step = cfg->Tnb[1] - cfg->Tnb[0];
    if (!(step >= 1.0) || !(step < 2147483647.0))
        return set_err(err_, RC_E_INVALID, "coupling Tnb step must be >= 1 K (linear_int divides by int(step))");
    memset(&a, 0, sizeof(a));
    a.stefan = cfg->stefan;
    a.Tin = cfg->Tin;
    a.Tin4 = pow(cfg->Tin, 4.0);
    a.Height = cfg->Height;
    a.underrelax = cfg->underrelax;
    a.imax = p.imax;
    a.jmax = p.jmax;
    a.kloc = c->kloc;
    a.jstart = cfg->jstart;
    a.jn = cfg->jend - cfg->jstart + 1;
    a.west = p.calcwalls && p.adiabw;
    a.east = p.calcwalls && p.adiabe;
    a.nT = cfg->nTemp;
    a.dT = (int)step;
    a.Mnx = Impl<float>::magic((unsigned long long)(p.imax + 2));
    a.Mjn = Impl<float>::magic((unsigned long long)a.jn);
    a.MdT = Impl<float>::magic((unsigned long long)a.dT);
    for (int t = 0; t < cfg->nTemp; ++t) {
        a.Tnb[t] = cfg->Tnb[t];
        a.kP[t] = cfg->kP[t];
    }
    for (int t = 0; t + 1 < cfg->nTemp; ++t) a.slope[t] = (a.kP[t + 1] - a.kP[t]) / (a.Tnb[t + 1] - a.Tnb[t]);
    return RC_OK;
}

SlotCommon *slot_of(rc_ctx *c, rc_ticket t) {
    SlotCommon *sp = nullptr;
    with_impl(c, [&](auto &im) {
        sp = im.find_slot(t);
        return 0;
    });
    return sp;
}

int launch_dns(const rc_ctx *c, const DnsArgs &a, cudaStream_t st, std::string *err_) {
    RC_FAILPOINT("dns");
    // every block resident at once: the SMs' worth of blocks, at most one
    // cell per thread
    static int per_sm = 0;
    if (!per_sm) {
        RC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dns_source, 256, 0));
        per_sm = std::max(per_sm, 1);
    }
    const long long n = (long long)(a.imax + 2) * a.jn * a.kloc;
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)c->num_sms * per_sm));
    k_dns_source<<<grid, 256, 0, st>>>(a);
    RC_CK(cudaGetLastError());
    return RC_OK;
}

size_t pencil_cells(const DnsArgs &a) { return (size_t)(a.imax + 2) * (a.jn + 2) * (a.kloc + 2); }
size_t out_cells(const DnsArgs &a) { return (size_t)(a.imax + 2) * a.jn * a.kloc; }

// memcpy split over up to 8 host threads (parts of >= 4 MB): one thread
// does not keep up with the PCIe copy engines.
void par_copy(void *dst, const void *src, size_t bytes) {
    const size_t min_part = (size_t)4 << 20;
    const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 8u));
    const size_t nt = std::max<size_t>(1, std::min<size_t>(hw, bytes / min_part));
    if (nt <= 1) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t part = ((bytes + nt - 1) / nt + 63) & ~(size_t)63;
    std::vector<std::thread> th;
    for (size_t i = 1; i < nt; ++i) {
        const size_t o = i * part;
        if (o >= bytes) break;
        th.emplace_back([=] { memcpy((char *)dst + o, (const char *)src + o, std::min(part, bytes - o)); });
    }
    memcpy(dst, src, std::min(part, bytes));
    for (auto &x : th) x.join();
}

}  // namespace

extern "C" {

int rc_dns_source(rc_ctx *c, rc_ticket t, const rc_dns_coupling *cfg, const double *T1, double *Qnew, double *Varnew,
                  double *Knew, double *Gnew, long long *n_clamped) {
    Range nv("rc_dns_source");
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    std::string *err_ = &c->err;
    if (!T1 || !Qnew || !Varnew || !Knew || !Gnew) return set_err(err_, RC_E_INVALID, "NULL array");
    cudaSetDevice(c->device);
    DnsArgs a;
    int rc = dns_args(c, cfg, a, err_);
    if (rc) return rc;
    SlotCommon *sp = slot_of(c, t);
    if (!sp) return set_err(err_, RC_E_STATE, "unknown or already collected ticket");
    SlotCommon &s = *sp;
    const size_t np = pencil_cells(a), no = out_cells(a);
    if (c->dns_cap < np + 4 * no) {
        if (c->d_dns) cudaFree(c->d_dns);
        c->d_dns = nullptr;
        c->dns_cap = 0;
        RC_CK(cudaMalloc((void **)&c->d_dns, (np + 4 * no) * sizeof(double)));
        c->dns_cap = np + 4 * no;
    }
    if (c->dns_hcap < np + 4 * no) {
        if (c->h_dns) cudaFreeHost(c->h_dns);
        c->h_dns = nullptr;
        c->dns_hcap = 0;
        RC_CK(cudaHostAlloc((void **)&c->h_dns, (np + 4 * no) * sizeof(double), cudaHostAllocDefault));
        c->dns_hcap = np + 4 * no;
    }
    if (!c->d_dns_n) RC_CK(cudaMalloc((void **)&c->d_dns_n, sizeof(unsigned long long)));
    double *dT1 = c->d_dns, *dQ = dT1 + np, *dV = dQ + no, *dK = dV + no, *dG = dK + no;
    a.Qc = s.d_Qc;
    a.Sc = s.d_Sc;
    a.Wq = s.d_Wq;
    a.Ws = s.d_Ws;
    a.T1 = dT1;
    a.Qnew = dQ;
    a.Varnew = dV;
    a.Knew = dK;
    a.Gnew = dG;
    a.n_clamped = c->d_dns_n;
    // T1 through the pinned staging buffer (the field is staged while the
    // solve may still run), then the kernel; each output array comes back
    // into the staging buffer and is copied out while the next one is in
    // flight
    double *hT1 = c->h_dns, *hOut = c->h_dns + np;
    par_copy(hT1, T1, np * sizeof(double));
    RC_CK(cudaEventSynchronize(s.e1));
    s.state = 2;
    RC_CK(cudaMemcpyAsync(dT1, hT1, np * sizeof(double), cudaMemcpyHostToDevice, s.st));
    RC_CK(cudaMemsetAsync(c->d_dns_n, 0, sizeof(unsigned long long), s.st));
    rc = launch_dns(c, a, s.st, err_);
    if (rc) return rc;
    cudaEvent_t ev[4] = {};
    double *const dst[4] = {Qnew, Varnew, Knew, Gnew};
    for (int q = 0; q < 4 && !rc; ++q) {
        if (cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming) != cudaSuccess ||
            cudaMemcpyAsync(hOut + q * no, dQ + q * no, no * sizeof(double), cudaMemcpyDeviceToHost, s.st) !=
                cudaSuccess ||
            cudaEventRecord(ev[q], s.st) != cudaSuccess)
            rc = set_err(err_, RC_E_CUDA, "staging the DNS source terms failed");
    }
    for (int q = 0; q < 4 && !rc; ++q) {
        if (cudaEventSynchronize(ev[q]) != cudaSuccess) rc = set_err(err_, RC_E_CUDA, "DNS source copy failed");
        else par_copy(dst[q], hOut + q * no, no * sizeof(double));
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (rc) return rc;
    unsigned long long nc = 0;
    RC_CK(cudaMemcpyAsync(&nc, c->d_dns_n, sizeof(nc), cudaMemcpyDeviceToHost, s.st));
    RC_CK(cudaStreamSynchronize(s.st));
    if (n_clamped) *n_clamped = (long long)nc;
    const int status = s.h_sc->status;
    s.state = 0;
    s.ticket = -1;
    if (status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values");
    return RC_OK;
}

int rc_dns_source_device(rc_ctx *c, rc_ticket t, const rc_dns_coupling *cfg, const double *T1_dev, double *Qnew_dev,
                         double *Varnew_dev, double *Knew_dev, double *Gnew_dev, unsigned long long *n_clamped_dev,
                         void *stream) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    std::string *err_ = &c->err;
    if (!T1_dev || !Qnew_dev || !Varnew_dev || !Knew_dev || !Gnew_dev)
        return set_err(err_, RC_E_INVALID, "NULL array");
    cudaSetDevice(c->device);
    DnsArgs a;
    int rc = dns_args(c, cfg, a, err_);
    if (rc) return rc;
    SlotCommon *sp = slot_of(c, t);
    if (!sp) return set_err(err_, RC_E_STATE, "unknown or already collected ticket");
    SlotCommon &s = *sp;
    a.Qc = s.d_Qc;
    a.Sc = s.d_Sc;
    a.Wq = s.d_Wq;
    a.Ws = s.d_Ws;
    a.T1 = T1_dev;
    a.Qnew = Qnew_dev;
    a.Varnew = Varnew_dev;
    a.Knew = Knew_dev;
    a.Gnew = Gnew_dev;
    a.n_clamped = n_clamped_dev;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s.st;
    if (st != s.st) RC_CK(cudaStreamWaitEvent(st, s.e1, 0));
    rc = launch_dns(c, a, st, err_);
    if (rc) return rc;
    if (st != s.st) {
        // the slot's next solve overwrites the results this kernel reads
        if (!s.e_dns) RC_CK(cudaEventCreateWithFlags(&s.e_dns, cudaEventDisableTiming));
        RC_CK(cudaEventRecord(s.e_dns, st));
        RC_CK(cudaStreamWaitEvent(s.st, s.e_dns, 0));
    }
    return RC_OK;
}

}  // extern "C"
