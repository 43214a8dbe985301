// rc_slab.cpp -- one solve over several GPUs from C: the reference's z-slab
// decomposition (mc_gpu_noint.cu:95-98, zstart / p_col) with the field
// broadcast from rank 0 and the slabs' results all-gathered over NCCL, so
// every rank ends with the whole solution (the reference's DNS combines the
// slabs with an MPI_Allreduce, fixvar.f:202-203).
//
// NCCL is loaded with dlopen when the first id or communicator is made, so
// the library itself does not depend on it.  Communicators are
// non-blocking: every wait (joining the group, each collective) polls with a
// deadline, and a group that misses it is aborted rather than left hanging.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>

#include "rc_host.h"

using rc_detail::set_err;

namespace {

struct NcclApi {
    bool ok = false;
    std::string why;  // why loading failed
    decltype(&ncclGetVersion) GetVersion = nullptr;
    decltype(&ncclGetUniqueId) GetUniqueId = nullptr;
    decltype(&ncclCommInitRankConfig) CommInitRankConfig = nullptr;
    decltype(&ncclCommGetAsyncError) CommGetAsyncError = nullptr;
    decltype(&ncclCommFinalize) CommFinalize = nullptr;
    decltype(&ncclCommDestroy) CommDestroy = nullptr;
    decltype(&ncclCommAbort) CommAbort = nullptr;
    decltype(&ncclBroadcast) Broadcast = nullptr;
    decltype(&ncclAllGather) AllGather = nullptr;
    decltype(&ncclGroupStart) GroupStart = nullptr;
    decltype(&ncclGroupEnd) GroupEnd = nullptr;
    decltype(&ncclGetErrorString) GetErrorString = nullptr;
};

// The process's NCCL: the file RC_NCCL_LIBRARY names, else libnccl.so.2
// (in a process that has already loaded an NCCL under that soname, e.g.
// through PyTorch, the dynamic loader returns that one).
const NcclApi &nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *env = getenv("RC_NCCL_LIBRARY");
        const char *name = (env && *env) ? env : "libnccl.so.2";
        void *h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            const char *e = dlerror();
            api.why = std::string("cannot load NCCL (") + name + "): " + (e ? e : "unknown error");
            return;
        }
        bool all = true;
        auto sym = [&](auto &fn, const char *s) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, s));
            if (!fn) {
                all = false;
                if (api.why.empty()) api.why = std::string("NCCL library lacks ") + s;
            }
        };
        sym(api.GetVersion, "ncclGetVersion");
        sym(api.GetUniqueId, "ncclGetUniqueId");
        sym(api.CommInitRankConfig, "ncclCommInitRankConfig");
        sym(api.CommGetAsyncError, "ncclCommGetAsyncError");
        sym(api.CommFinalize, "ncclCommFinalize");
        sym(api.CommDestroy, "ncclCommDestroy");
        sym(api.CommAbort, "ncclCommAbort");
        sym(api.Broadcast, "ncclBroadcast");
        sym(api.AllGather, "ncclAllGather");
        sym(api.GroupStart, "ncclGroupStart");
        sym(api.GroupEnd, "ncclGroupEnd");
        sym(api.GetErrorString, "ncclGetErrorString");
        api.ok = all;
    });
    return api;
}

using Clock = std::chrono::steady_clock;

}  // namespace

struct rc_slab_comm {
    int device = 0, nranks = 1, rank = 0;
    double timeout_s = 300.0;
    ncclComm_t comm = nullptr;
    cudaStream_t st = nullptr;
    bool dead = false;  // aborted: only rc_slab_comm_destroy is valid
    // device buffers, grown on demand: wall-flux staging (this rank's
    // [4][kloc][jmax] -- qw west, qw east, vw west, vw east -- followed by
    // every rank's, gathered), and stand-ins for arrays the caller passes in
    // host memory (field, q64, var64, qw64, vw64)
    struct Buf {
        void *p = nullptr;
        size_t cap = 0;
    };
    Buf walls, stage[5];
    std::string err;
};

namespace {

int fail(rc_slab_comm *c, int code, const std::string &m) { return set_err(c ? &c->err : nullptr, code, m); }

std::string nccl_msg(const char *what, ncclResult_t r) {
    return std::string(what) + ": " + nccl().GetErrorString(r);
}

// Aborts the group after a timeout or an asynchronous NCCL error.
int abort_group(rc_slab_comm *c, int code, const std::string &m) {
    if (c->comm && !c->dead) nccl().CommAbort(c->comm);
    c->comm = nullptr;
    c->dead = true;
    return fail(c, code, m);
}

// Waits until the communicator has no call in progress (a non-blocking
// communicator returns ncclInProgress from calls it has not finished).
int wait_comm(rc_slab_comm *c, const Clock::time_point deadline, const char *what) {
    for (;;) {
        ncclResult_t a = ncclSuccess;
        const ncclResult_t r = nccl().CommGetAsyncError(c->comm, &a);
        if (r != ncclSuccess) return abort_group(c, RC_E_CUDA, nccl_msg(what, r));
        if (a == ncclSuccess) return RC_OK;
        if (a != ncclInProgress) return abort_group(c, RC_E_CUDA, nccl_msg(what, a));
        if (Clock::now() > deadline)
            return abort_group(c, RC_E_TIMEOUT, std::string(what) + ": timed out; the group is aborted");
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
}

// The result of an NCCL call on a non-blocking communicator.
int after_call(rc_slab_comm *c, ncclResult_t r, const Clock::time_point deadline, const char *what) {
    if (r == ncclInProgress) return wait_comm(c, deadline, what);
    if (r != ncclSuccess) return abort_group(c, RC_E_CUDA, nccl_msg(what, r));
    return RC_OK;
}

// Waits for the communicator's stream (its collectives) with the deadline.
int wait_stream(rc_slab_comm *c, const Clock::time_point deadline, const char *what) {
    for (;;) {
        const cudaError_t e = cudaStreamQuery(c->st);
        if (e == cudaSuccess) return RC_OK;
        if (e != cudaErrorNotReady) return fail(c, RC_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        ncclResult_t a = ncclSuccess;
        nccl().CommGetAsyncError(c->comm, &a);
        if (a != ncclSuccess && a != ncclInProgress) return abort_group(c, RC_E_CUDA, nccl_msg(what, a));
        if (Clock::now() > deadline)
            return abort_group(c, RC_E_TIMEOUT, std::string(what) + ": timed out; the group is aborted");
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

// Grows b to at least `bytes` of device memory.
int ensure(rc_slab_comm *c, rc_slab_comm::Buf &b, size_t bytes, const char *what) {
    if (bytes <= b.cap) return RC_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    const cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) return fail(c, RC_E_NOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    b.cap = bytes;
    return RC_OK;
}

// Where an array lives: 1 device memory of `device` (or managed memory),
// which NCCL and the solver use as is; 0 host memory (staged); -1 device
// memory of another GPU (refused: it would be read across devices).
int placement(const void *ptr, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();  // a plain host pointer on an old runtime
        return 0;
    }
    if (a.type == cudaMemoryTypeManaged) return 1;
    if (a.type == cudaMemoryTypeDevice) return a.device == device ? 1 : -1;
    return 0;
}

Clock::time_point deadline_of(const rc_slab_comm *c) {
    return Clock::now() + std::chrono::microseconds((long long)(c->timeout_s * 1e6));
}

}  // namespace

extern "C" {

int rc_slab_range(int kmax, int nranks, int rank, int *kloc, int *zstart) {
    if (kmax < 1 || nranks < 1 || rank < 0 || rank >= nranks)
        return set_err(nullptr, RC_E_INVALID, "rank outside the group, or an empty grid");
    if (kmax % nranks)
        return set_err(nullptr, RC_E_INVALID,
                       "kmax = " + std::to_string(kmax) + " is not a multiple of the group size " +
                           std::to_string(nranks));
    const int kl = kmax / nranks;
    if (kloc) *kloc = kl;
    if (zstart) *zstart = rank * kl + 1;
    return RC_OK;
}

int rc_slab_unique_id(void *id) {
    if (!id) return set_err(nullptr, RC_E_INVALID, "NULL id");
    const NcclApi &n = nccl();
    if (!n.ok) return set_err(nullptr, RC_E_NOTFOUND, n.why);
    ncclUniqueId uid;
    const ncclResult_t r = n.GetUniqueId(&uid);
    if (r != ncclSuccess) return set_err(nullptr, RC_E_CUDA, nccl_msg("ncclGetUniqueId", r));
    static_assert(sizeof(uid) == RC_SLAB_ID_BYTES, "NCCL unique id size");
    memcpy(id, &uid, sizeof uid);
    return RC_OK;
}

int rc_slab_comm_create(int device, int nranks, int rank, const void *id, double timeout_s, rc_slab_comm **out) {
    if (!id || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    if (nranks < 1 || rank < 0 || rank >= nranks) return set_err(nullptr, RC_E_INVALID, "rank outside the group");
    const NcclApi &n = nccl();
    if (!n.ok) return set_err(nullptr, RC_E_NOTFOUND, n.why);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_err(nullptr, RC_E_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return set_err(nullptr, RC_E_INVALID, "device index out of range");
    if ((e = cudaSetDevice(device)) != cudaSuccess) return set_err(nullptr, RC_E_CUDA, cudaGetErrorString(e));
    auto *c = new rc_slab_comm();
    c->device = device;
    c->nranks = nranks;
    c->rank = rank;
    c->timeout_s = timeout_s > 0 ? timeout_s : 300.0;
    if ((e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) != cudaSuccess) {
        delete c;
        return set_err(nullptr, RC_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    ncclUniqueId uid;
    memcpy(&uid, id, sizeof uid);
    const auto deadline = deadline_of(c);
    const ncclResult_t r = n.CommInitRankConfig(&c->comm, nranks, uid, rank, &cfg);
    int rc = RC_OK;
    if (r != ncclSuccess && r != ncclInProgress)
        rc = c->comm ? abort_group(c, RC_E_CUDA, nccl_msg("ncclCommInitRank", r))
                     : set_err(nullptr, RC_E_CUDA, nccl_msg("ncclCommInitRank", r));
    else if (r == ncclInProgress || c->comm) rc = wait_comm(c, deadline, "joining the group");
    if (rc != RC_OK) {
        const std::string m = c->err.empty() ? rc_detail::g_err : c->err;
        rc_slab_comm_destroy(c);
        return set_err(nullptr, rc, m);
    }
    *out = c;
    return RC_OK;
}

int rc_slab_solve(rc_slab_comm *c, rc_ctx *ctx, float *T, double *q64, double *var64, double *qw64,
                  double *vw64) {
    if (!c || !ctx || !T || !q64 || !var64) return fail(c, RC_E_INVALID, "NULL argument");
    if (c->dead) return fail(c, RC_E_STATE, "the group was aborted after an earlier failure");
    rc_params p;
    int dev = -1;
    int rc = rc_get_params(ctx, &p, &dev);
    if (rc) return fail(c, rc, rc_detail::g_err);
    if (dev != c->device) return fail(c, RC_E_INVALID, "the context lives on another device than the communicator");
    if (p.p_col != c->nranks)
        return fail(c, RC_E_INVALID,
                    "the context's p_col (" + std::to_string(p.p_col) + ") differs from the group size " +
                        std::to_string(c->nranks));
    int kloc = 0, zstart = 0;
    if ((rc = rc_slab_range(p.kmax, c->nranks, c->rank, &kloc, &zstart))) return fail(c, rc, rc_detail::g_err);
    cudaSetDevice(c->device);
    const NcclApi &n = nccl();
    const size_t nT = (size_t)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
    const size_t ncell = (size_t)p.imax * p.jmax * kloc;  // cells of one slab
    const size_t nw = (size_t)p.jmax * kloc;              // cells of one wall in one slab
    const size_t nwall = (size_t)2 * p.jmax * p.kmax;     // both walls, whole solution
    if ((rc = ensure(c, c->walls, (size_t)4 * nw * (1 + c->nranks) * sizeof(double), "wall staging"))) return rc;
    double *wl = static_cast<double *>(c->walls.p), *wg = wl + 4 * nw;
    // arrays in host memory go through device stand-ins
    void *user[5] = {T, q64, var64, qw64, vw64};
    const size_t bytes[5] = {nT * sizeof(float), ncell * c->nranks * sizeof(double),
                             ncell * c->nranks * sizeof(double), nwall * sizeof(double), nwall * sizeof(double)};
    void *dv[5];
    bool staged[5];
    for (int a = 0; a < 5; ++a) {
        const int where = user[a] ? placement(user[a], c->device) : 1;
        if (where < 0) return fail(c, RC_E_INVALID, "an array lives on another GPU than the communicator's");
        staged[a] = where == 0;
        dv[a] = user[a];
        if (staged[a]) {
            if ((rc = ensure(c, c->stage[a], bytes[a], "staging of a host array"))) return rc;
            dv[a] = c->stage[a].p;
        }
    }
    float *Td = static_cast<float *>(dv[0]);
    double *qd = static_cast<double *>(dv[1]), *vd = static_cast<double *>(dv[2]);
    double *qwd = static_cast<double *>(dv[3]), *vwd = static_cast<double *>(dv[4]);

    // the field: rank 0's into every rank's buffer
    auto deadline = deadline_of(c);
    if (staged[0] && c->rank == 0) {
        const cudaError_t e = cudaMemcpyAsync(Td, T, bytes[0], cudaMemcpyHostToDevice, c->st);
        if (e != cudaSuccess) return fail(c, RC_E_CUDA, std::string("field copy: ") + cudaGetErrorString(e));
    }
    if ((rc = after_call(c, n.Broadcast(Td, Td, nT, ncclFloat, 0, c->comm, c->st), deadline, "ncclBroadcast")))
        return rc;
    if ((rc = wait_stream(c, deadline, "field broadcast"))) return rc;

    // this rank's slab, written where it lies in the whole solution; a
    // failure here is reported after the gathers, which every rank makes
    rc_ticket t = 0;
    int solve_rc = rc_solve_device_async(ctx, Td, zstart, &t);
    if (solve_rc == RC_OK)
        solve_rc = rc_collect_device(ctx, t, qd + (size_t)c->rank * ncell, vd + (size_t)c->rank * ncell, wl,
                                     wl + 2 * nw);
    std::string solve_msg;
    if (solve_rc != RC_OK) {
        char buf[512];
        rc_last_error(ctx, buf, sizeof buf);
        solve_msg = buf;
    }

    // every slab to every rank (in place for the cell arrays)
    deadline = deadline_of(c);
    if ((rc = after_call(c, n.GroupStart(), deadline, "ncclGroupStart"))) return rc;
    ncclResult_t r = n.AllGather(qd + (size_t)c->rank * ncell, qd, ncell, ncclFloat64, c->comm, c->st);
    if (r == ncclSuccess || r == ncclInProgress)
        r = n.AllGather(vd + (size_t)c->rank * ncell, vd, ncell, ncclFloat64, c->comm, c->st);
    if (r == ncclSuccess || r == ncclInProgress) r = n.AllGather(wl, wg, 4 * nw, ncclFloat64, c->comm, c->st);
    const ncclResult_t r_end = n.GroupEnd();
    if ((rc = after_call(c, r != ncclSuccess && r != ncclInProgress ? r : r_end, deadline, "ncclAllGather")))
        return rc;
    // walls: gathered [rank][4][kloc][jmax] -> [wall][kmax][jmax], one
    // strided copy per output array and wall
    for (int a = 0; a < 2; ++a) {
        double *dst = a ? vwd : qwd;
        if (!dst) continue;
        for (int w = 0; w < 2; ++w) {
            const cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)w * p.kmax * p.jmax, nw * sizeof(double),
                                                    wg + (size_t)(2 * a + w) * nw, 4 * nw * sizeof(double),
                                                    nw * sizeof(double), c->nranks, cudaMemcpyDeviceToDevice, c->st);
            if (e != cudaSuccess) return fail(c, RC_E_CUDA, std::string("wall copy: ") + cudaGetErrorString(e));
        }
    }
    // host arrays back (the field too on the ranks that received it)
    for (int a = 0; a < 5; ++a) {
        if (!staged[a] || (a == 0 && c->rank == 0)) continue;
        const cudaError_t e = cudaMemcpyAsync(user[a], dv[a], bytes[a], cudaMemcpyDeviceToHost, c->st);
        if (e != cudaSuccess) return fail(c, RC_E_CUDA, std::string("result copy: ") + cudaGetErrorString(e));
    }
    if ((rc = wait_stream(c, deadline, "result gather"))) return rc;
    if (solve_rc != RC_OK) return fail(c, solve_rc, "slab solve on rank " + std::to_string(c->rank) + ": " + solve_msg);
    return RC_OK;
}

int rc_slab_last_error(const rc_slab_comm *c, char *buf, size_t len) {
    const std::string &m = c ? c->err : rc_detail::g_err;
    if (buf && len) snprintf(buf, len, "%s", m.c_str());
    return RC_OK;
}

int rc_slab_comm_destroy(rc_slab_comm *c) {
    if (!c) return RC_OK;
    cudaSetDevice(c->device);
    int rc = RC_OK;
    if (c->comm && !c->dead) {
        const NcclApi &n = nccl();
        const auto deadline = deadline_of(c);
        rc = after_call(c, n.CommFinalize(c->comm), deadline, "ncclCommFinalize");
        if (rc == RC_OK && c->comm) {
            n.CommDestroy(c->comm);
            c->comm = nullptr;
        }
    }
    if (c->walls.p) cudaFree(c->walls.p);
    for (auto &b : c->stage)
        if (b.p) cudaFree(b.p);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return rc;
}

}  // extern "C"
