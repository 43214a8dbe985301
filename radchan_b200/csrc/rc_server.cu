// rc_server.cu -- continuous-batching solve server.
//
// The reference solves one field per mc_gpu_ call, synchronously
// (src/montecarlo/mc_gpu_noint.cu:659-1013).  The server accepts many
// independent solve requests (temperature field, parameter set, table set,
// photmax or a target relative standard deviation of max|Q|) and keeps one
// GPU busy with all of them at once:
//
//   * admission in arrival order, bounded by max_inflight and a device-memory
//     budget; every admitted request takes a pooled solver context whose
//     grid, tables and buffers stay resident between requests of the same
//     problem class (everything but photmax and the seed equal);
//   * one scheduler thread drives the GPU in quanta: a quantum is one
//     persistent march launch whose work queue holds tiles of every running
//     request -- by default the requests with the least remaining work
//     first, above a floor share for everyone (or equal shares, processor
//     sharing) -- so a request that arrives while long solves run joins the
//     next quantum instead of queueing behind them;
//   * quanta go round-robin to eight streams, so a quantum's tail (its
//     longest rays: in near-transparent bands a ray can take up to the last
//     level's step budget, maxs, tens of milliseconds) overlaps the next
//     quanta instead of idling the GPU; the prelude of each quantum (set-up
//     kernels, descriptor copies) is chained by events so it stays ordered;
//   * the request whose last tiles ran in a quantum gets its tally and the
//     scalar copy-back on a separate stream, after every quantum that may
//     still hold its tiles.
//
// Results are bit-identical to the same request solved alone by a context:
// every bundle's history depends only on (seed, cell, replicate, bundle),
// a tile of 32 work items is always marched inside one launch, and partial
// sums are combined in a fixed order by the tally.
//
// A request with a tolerance first runs a pilot solve of 64 bundles per cell
// (skipped once a request of the same problem class has calibrated the
// bundle count), then the solve with photmax = n0 (s0 / tol)^2, as the
// relative Monte Carlo standard deviation falls as photmax^-1/2.
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

#include "rc_impl.cuh"

using namespace rc_detail;

namespace rc_detail {

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum SrvStage : int { ST_QUEUED = 0, ST_PILOT = 1, ST_MAIN = 2, ST_DONE = 3, ST_FAILED = 4 };
enum SrvPhase : int { PH_PREPARE = 0, PH_MARCH = 1, PH_TALLY = 2 };

struct SrvReq {
    int64_t id = 0;
    rc_params p;
    int table_set = -1;
    std::vector<float> T;
    int zstart = 1;
    float tol = 0.f;
    int stage = ST_QUEUED;
    int phase = PH_PREPARE;
    bool published = false;  // result visible to rc_server_wait (guarded by the server mutex)
    bool cancel = false;     // rc_server_cancel on a running request (guarded by the server mutex)
    double t_submit = 0, t_admit = 0, t_done = 0;
    rc_ctx *ctx = nullptr;
    Slot<float> *slot = nullptr;
    std::string key;
    // particle scattering of the request's table set at submit time (null: none)
    std::shared_ptr<const ScatterSet> scatter;
    long long tiles = 0, next_tile = 0;
    int photmax = 0;
    float rel_std = 0.f;
    int status = RC_OK;
    std::string err;
    cudaEvent_t ev = nullptr;
    std::vector<float> Q, S;
};

struct PoolCtx {
    rc_ctx *ctx;
    size_t bytes;
    std::string key;
    bool busy;
};

// Quantum size when none is set: a 32nd of the running requests' remaining
// tiles, between kQuantumTiles (16.8M bundles at 4 rays per thread, about
// 2 ms of march) and kQuantumMax.  Small backlogs keep quanta short, so a new
// request joins the device soon; a large backlog (many solves submitted at
// once) pays fewer quantum preludes and tails per solve.
constexpr long long kQuantumTiles = 131072;
constexpr long long kQuantumMax = 4 * kQuantumTiles;
constexpr long long kMinShare = 4096;
constexpr int kPilotPhotmax = 64;
constexpr int kMaxPhotmax = 1 << 20;

}  // namespace rc_detail

struct rc_server {
    int device = 0;
    double budget = 0;
    int max_inflight = 8;
    long long quantum_tiles = 0;  // 0: sized from the backlog (kQuantumTiles .. kQuantumMax)
    int policy = RC_SCHED_SRPT;
    long long quanta = 0;
    std::vector<std::unique_ptr<TableSet>> tables;  // stable addresses: appended while the worker reads
    // particle scattering per table set (-1: grey requests), replaced whole
    // by rc_server_set_scattering; a request keeps the one current at submit
    std::map<int, std::shared_ptr<const ScatterSet>> scatter;
    std::map<int, int> scatter_gen;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SrvReq *> queue;
    std::map<int64_t, std::unique_ptr<SrvReq>> reqs;
    std::vector<SrvReq *> running;
    std::vector<PoolCtx> pool;
    std::map<std::string, std::pair<int, float>> calib;  // class -> (photmax, rel std)
    int64_t next_id = 1;
    double hbm_in_use = 0;
    double solves_done = 0, busy_s = 0;
    bool stop = false;
    std::thread worker;
    cudaStream_t st = nullptr;  // tallies and result copies
    // quantum streams and launch buffers, one set per parity
    static constexpr int kNQ = 8;
    cudaStream_t qst[kNQ] = {};
    int cap = 0;
    DSolve<float> *d_solves[kNQ] = {};
    long long *d_tiles[kNQ] = {};
    long long *d_base[kNQ] = {};
    long long *h_tiles[kNQ] = {};
    long long *h_base[kNQ] = {};
    unsigned long long *d_counter[kNQ] = {};
    cudaEvent_t pre_done[kNQ] = {};  // prelude (set-up, descriptors) of the parity's latest quantum done
    cudaEvent_t mend[kNQ] = {};      // march of the parity's latest quantum done
    bool q_used[kNQ] = {};
    int q_par = 0, last_par = -1;
    // the set-up chains of the requests a quantum starts run side by side on
    // these streams, forked from and joined back into the quantum's stream
    static constexpr int kSide = 16;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr, join[kSide] = {};
    double busy_since = -1.0;
    std::string err;
};

namespace rc_detail {

__global__ void k_set_tile_base(DSolve<float> *d, const long long *base, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i].tile_base = base[i];
}

// Problem class: everything that fixes a context's device layout.
std::string class_key(const rc_params &p, int table_set) {
    rc_params q = p;
    q.photmax = 0;
    q.seed = 0;
    std::string k((const char *)&q, sizeof(q));
    k += "/" + std::to_string(table_set);
    return k;
}

// Device bytes of one context (two slots, default 4 rays per thread):
// the allocations of Impl::init, the tables and the partial-sum array.
size_t context_bytes(const rc_params &p, int photmax) {
    const int kl = p.kmax / p.p_col;
    const double nfield = (double)(p.imax + 2) * (p.jmax + 2) * (p.kmax + 2);
    const double ncf = (double)p.imax * p.jmax * kl, nwc = 2.0 * p.jmax * kl;
    double slot = nfield * 4 + ncf * 24 + nwc * 24 + 2.0 * p.jmax * p.kmax * 2;
    for (int l = 0; l < p.grid_num; ++l) {
        slot += (double)p.maxi[l] * p.maxj[l] * p.maxk[l] * 2 + 2.0 * ((double)p.maxj[l] * p.maxk[l] + (double)p.maxi[l] * p.maxk[l] +
                                      (double)p.maxi[l] * p.maxj[l]) * 2;
    }
    const int nB = p.grey ? p.grey_nB : p.nB, nT = p.grey ? p.grey_nT : p.nT, nQ = p.grey ? 1 : p.nQ;
    const double tabs = (double)nB * nQ * nT * (4 + 4 + sizeof(KIRow<float>)) + (double)nB * nT * 8;
    if (p.grey) slot += (double)nT * nB * (4 + sizeof(KIRow<float>));
    const int rpt = 4;
    const long long nchunk = ((long long)std::max(photmax, 1) + rpt - 1) / rpt;
    const long long nparts = nchunk <= 32 ? 1 : (nchunk + 31) / 32;
    const double partial = (ncf + nwc) * p.nVar * (double)nparts * 8;
    return (size_t)(2 * slot + tabs + partial + (1 << 20));
}

// Relative standard deviation of max|Q|: the RMS sigma of the cells whose
// |Q| is within 10% of the maximum, over max|Q|.  Pooling those cells keeps
// the estimate stable when nVar (the replicates behind each sigma) is small.
float rel_std_maxq(const float *Qc, const float *Sc, size_t n) {
    float best = 0.f;
    for (size_t c = 0; c < n; ++c) best = std::max(best, fabsf(Qc[c]));
    if (!(best > 0.f)) return 0.f;
    double s2 = 0.0;
    long long m = 0;
    for (size_t c = 0; c < n; ++c)
        if (fabsf(Qc[c]) >= 0.9f * best) {
            s2 += (double)Sc[c] * Sc[c];
            ++m;
        }
    return (float)(std::sqrt(s2 / (double)m) / best);
}

int photmax_for(int n0, float s0, float tol) {
    const double want = (double)n0 * ((double)s0 / tol) * ((double)s0 / tol);
    return (int)std::min((double)kMaxPhotmax, std::max((double)kPilotPhotmax, std::ceil(want)));
}

}  // namespace rc_detail

namespace {

// ---- scheduler (worker thread)

int grow_quantum_buffers(rc_server *sv, int n) {
    std::string *err_ = &sv->err;
    if (n <= sv->cap) return RC_OK;
    for (int i = 0; i < rc_server::kNQ; ++i) RC_CK(cudaStreamSynchronize(sv->qst[i]));
    for (int i = 0; i < rc_server::kNQ; ++i) {
        if (sv->d_solves[i]) cudaFree(sv->d_solves[i]);
        if (sv->d_tiles[i]) cudaFree(sv->d_tiles[i]);
        if (sv->d_base[i]) cudaFree(sv->d_base[i]);
        if (sv->h_tiles[i]) cudaFreeHost(sv->h_tiles[i]);
        if (sv->h_base[i]) cudaFreeHost(sv->h_base[i]);
        sv->d_solves[i] = nullptr;
        sv->d_tiles[i] = sv->d_base[i] = sv->h_tiles[i] = sv->h_base[i] = nullptr;
    }
    sv->cap = 0;
    const int c = std::max(n, 64);
    for (int i = 0; i < rc_server::kNQ; ++i) {
        RC_CK(cudaMalloc((void **)&sv->d_solves[i], c * sizeof(DSolve<float>)));
        RC_CK(cudaMalloc((void **)&sv->d_tiles[i], (c + 1) * sizeof(long long)));
        RC_CK(cudaMalloc((void **)&sv->d_base[i], c * sizeof(long long)));
        RC_CK(cudaHostAlloc((void **)&sv->h_tiles[i], (c + 1) * sizeof(long long), cudaHostAllocDefault));
        RC_CK(cudaHostAlloc((void **)&sv->h_base[i], c * sizeof(long long), cudaHostAllocDefault));
    }
    sv->cap = c;
    return RC_OK;
}

size_t idle_bytes(const rc_server *sv) {
    size_t b = 0;
    for (const auto &pc : sv->pool)
        if (!pc.busy) b += pc.bytes;
    return b;
}

bool has_idle_context(const rc_server *sv, const std::string &key) {
    for (const auto &pc : sv->pool)
        if (!pc.busy && pc.key == key) return true;
    return false;
}

// Take a pooled context of the request's class, or create one (evicting
// idle contexts of other classes while over the budget).
int acquire_context(rc_server *sv, SrvReq *r) {
    for (auto &pc : sv->pool)
        if (!pc.busy && pc.key == r->key) {
            pc.busy = true;
            r->ctx = pc.ctx;
            return RC_OK;
        }
    const size_t need = context_bytes(r->p, std::max(r->photmax, kPilotPhotmax));
    for (size_t i = 0; i < sv->pool.size() && sv->hbm_in_use + need > sv->budget;) {
        if (!sv->pool[i].busy) {
            {
                std::lock_guard<std::mutex> lk(sv->mu);
                sv->hbm_in_use -= sv->pool[i].bytes;
            }
            rc_destroy(sv->pool[i].ctx);
            sv->pool.erase(sv->pool.begin() + i);
        } else {
            ++i;
        }
    }
    if (sv->hbm_in_use + need > sv->budget) return set_err(nullptr, RC_E_NOMEM, "HBM budget exhausted");
    rc_ctx *c = nullptr;
    int rc = rc_create(&r->p, sv->device, &c);
    if (rc) return rc;
    if (!r->p.grey) {
        rc_tables v;
        const TableSet *ts;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            ts = sv->tables[r->table_set].get();
        }
        ts->view(&v);
        rc = rc_set_tables(c, &v);
        if (rc) {
            const std::string m = c->err;
            rc_destroy(c);
            return set_err(nullptr, rc, m);
        }
    }
    if (r->scatter) {
        rc_scattering sv_view;
        r->scatter->view(&sv_view);
        rc = rc_set_scattering(c, &sv_view);
        if (rc) {
            const std::string m = c->err;
            rc_destroy(c);
            return set_err(nullptr, rc, m);
        }
    }
    sv->pool.push_back(PoolCtx{c, need, r->key, true});
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->hbm_in_use += need;
    r->ctx = c;
    return RC_OK;
}

void release_context(rc_server *sv, SrvReq *r) {
    for (auto &pc : sv->pool)
        if (pc.ctx == r->ctx) pc.busy = false;
    r->ctx = nullptr;
}

void fail(rc_server *sv, SrvReq *r, int code, const std::string &m) {
    r->status = code;
    r->err = m;
    r->stage = ST_FAILED;
    r->t_done = now_s();
    if (r->slot) r->slot->state = 0;
    r->slot = nullptr;
    if (r->ctx) release_context(sv, r);
}

// Budget share of a context whose partial-sum array grows with photmax.
void account_photmax(rc_server *sv, SrvReq *r) {
    for (auto &pc : sv->pool)
        if (pc.ctx == r->ctx) {
            const size_t b = context_bytes(r->p, r->photmax);
            if (b > pc.bytes) {
                std::lock_guard<std::mutex> lk(sv->mu);
                sv->hbm_in_use += (double)(b - pc.bytes);
                pc.bytes = b;
            }
        }
}

// Partial-sum array for the stage's photmax, from the stream-ordered
// allocator: a plain cudaFree would wait for every quantum in flight.  The
// old array's last users (marches and the tally of the previous stage) have
// finished: the host saw the tally's event.
int ensure_partial_async(rc_server *sv, SrvReq *r, cudaStream_t st) {
    std::string *err_ = &sv->err;
    Impl<float> &im = *static_cast<Impl<float> *>(r->ctx->impl);
    Slot<float> &s = *r->slot;
    const size_t need = im.partial_count(r->ctx->rpt);
    if (need <= s.partial_cap) return RC_OK;
    if (s.d_partial) RC_CK(cudaFreeAsync(s.d_partial, st));
    s.d_partial = nullptr;
    s.partial_cap = 0;
    RC_CK(cudaMallocAsync((void **)&s.d_partial, need * sizeof(double), st));
    s.partial_cap = need;
    return RC_OK;
}

// Field copy, set-up kernels and descriptor of the request's current stage.
int start_stage(rc_server *sv, SrvReq *r, cudaStream_t st) {
    Impl<float> &im = *static_cast<Impl<float> *>(r->ctx->impl);
    r->ctx->p.photmax = r->photmax;
    r->ctx->p.seed = r->p.seed;
    account_photmax(sv, r);
    int rc = ensure_partial_async(sv, r, st);
    if (rc) return rc;
    rc = im.prepare(*r->slot, nullptr, r->zstart, r->ctx->rpt, st);
    if (rc) return rc;
    r->tiles = r->slot->h_desc->n_tiles;
    r->next_tile = 0;
    r->phase = PH_MARCH;
    return RC_OK;
}

// Prelude and march of one quantum on stream qst[par]: equal shares of every
// marching request's remaining tiles in one persistent launch.  Set-up work
// of new stages was enqueued on the same stream just before.
int run_quantum(rc_server *sv, const std::vector<SrvReq *> &marching, int par) {
    Range nv("rc_server quantum");
    std::string *err_ = &sv->err;
    RC_FAILPOINT("quantum");
    const int n = (int)marching.size();
    cudaStream_t st = sv->qst[par];
    long long *ht = sv->h_tiles[par], *hb = sv->h_base[par];
    ht[0] = 0;
    long long qt;
    int policy;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        qt = sv->quantum_tiles;
        policy = sv->policy;
        sv->quanta++;
    }
    if (qt <= 0) {
        long long backlog = 0;
        for (int i = 0; i < n; ++i) backlog += marching[i]->tiles - marching[i]->next_tile;
        qt = std::min(kQuantumMax, std::max(kQuantumTiles, backlog / 32));
    }
    std::vector<long long> take(n, 0);
    if (policy == RC_SCHED_FAIR) {
        const long long share = std::max<long long>(qt / n, kMinShare);
        for (int i = 0; i < n; ++i) take[i] = std::min(share, marching[i]->tiles - marching[i]->next_tile);
    } else {
        // shortest remaining work first, with a floor of 1/8 of the quantum
        // shared by everyone so that long requests keep progressing
        long long budget = std::max(qt, kMinShare);
        const long long floor = std::max<long long>(budget / (8LL * n), 1);
        for (int i = 0; i < n; ++i) {
            take[i] = std::min(floor, marching[i]->tiles - marching[i]->next_tile);
            budget -= take[i];
        }
        std::vector<int> order(n);
        for (int i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return marching[a]->tiles - marching[a]->next_tile < marching[b]->tiles - marching[b]->next_tile;
        });
        for (int i : order) {
            if (budget <= 0) break;
            const long long more = std::min(budget, marching[i]->tiles - marching[i]->next_tile - take[i]);
            take[i] += more;
            budget -= more;
        }
    }
    int rpt_max = 1;
    for (int i = 0; i < n; ++i) {
        SrvReq *r = marching[i];
        hb[i] = r->next_tile;
        ht[i + 1] = ht[i] + take[i];
        r->next_tile += take[i];
        rpt_max = std::max(rpt_max, r->ctx->rpt);
        RC_CK(cudaMemcpyAsync(sv->d_solves[par] + i, r->slot->d_desc, sizeof(DSolve<float>),
                              cudaMemcpyDeviceToDevice, st));
    }
    RC_CK(cudaMemcpyAsync(sv->d_tiles[par], ht, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
    RC_CK(cudaMemcpyAsync(sv->d_base[par], hb, n * sizeof(long long), cudaMemcpyHostToDevice, st));
    k_set_tile_base<<<(n + 127) / 128, 128, 0, st>>>(sv->d_solves[par], sv->d_base[par], n);
    RC_CK(cudaGetLastError());
    RC_CK(cudaEventRecord(sv->pre_done[par], st));
    if (ht[n] > 0) {
        Impl<float> &im0 = *static_cast<Impl<float> *>(marching[0]->ctx->impl);
        int scat = 0;  // the scattering variant of the march when any request's medium scatters
        for (int i = 0; i < n; ++i)
            if (static_cast<Impl<float> *>(marching[i]->ctx->impl)->nA > 0) scat = 1;
        const int rc = im0.launch_march(sv->d_solves[par], sv->d_tiles[par], n, ht[n], sv->d_counter[par],
                                        marching[0]->ctx->block, rpt_max, st, 0, nullptr, scat);
        if (rc) return set_err(err_, rc, marching[0]->ctx->err);
    }
    RC_CK(cudaEventRecord(sv->mend[par], st));
    return RC_OK;
}

// Tallies of the requests whose last tiles were just issued, on the tally
// stream after every quantum in flight (any of them may hold their tiles).
int enqueue_tallies(rc_server *sv, const std::vector<SrvReq *> &marching) {
    Range nv("rc_server tallies");
    std::string *err_ = &sv->err;
    bool waited = false;
    for (SrvReq *r : marching) {
        if (r->next_tile < r->tiles) continue;
        if (!waited) {
            for (int q = 0; q < rc_server::kNQ; ++q)
                if (sv->q_used[q]) RC_CK(cudaStreamWaitEvent(sv->st, sv->mend[q], 0));
            waited = true;
        }
        Impl<float> &im = *static_cast<Impl<float> *>(r->ctx->impl);
        int rc = im.launch_tally(r->slot->d_desc, r->slot->d_out, 1, im.tally_cells(), sv->st);
        if (rc) return set_err(err_, rc, r->ctx->err);
        RC_CK(cudaMemcpyAsync(r->slot->h_sc, r->slot->d_sc, sizeof(DScalars), cudaMemcpyDeviceToHost, sv->st));
        RC_CK(cudaEventRecord(r->ev, sv->st));
        r->phase = PH_TALLY;
    }
    return RC_OK;
}

// A request whose tally finished: pilot -> main solve, or results -> done.
void finish_stage(rc_server *sv, SrvReq *r) {
    Impl<float> &im = *static_cast<Impl<float> *>(r->ctx->impl);
    Slot<float> &s = *r->slot;
    const size_t ncf = (size_t)r->p.imax * r->p.jmax * r->ctx->kloc;
    if (s.h_sc->status & 2) {
        fail(sv, r, RC_E_RANGE, "temperature field contains non-finite values");
        return;
    }
    if (r->stage == ST_PILOT) {
        if (cudaMemcpyAsync(s.h_Qc, s.d_Qc, ncf * sizeof(float), cudaMemcpyDeviceToHost, s.st) != cudaSuccess ||
            cudaMemcpyAsync(s.h_Sc, s.d_Sc, ncf * sizeof(float), cudaMemcpyDeviceToHost, s.st) != cudaSuccess ||
            cudaStreamSynchronize(s.st) != cudaSuccess) {
            fail(sv, r, RC_E_CUDA, "pilot copy failed");
            return;
        }
        const float s0 = rel_std_maxq(s.h_Qc, s.h_Sc, ncf);
        r->photmax = s0 > 0 ? photmax_for(r->photmax, s0, r->tol) : kPilotPhotmax;
        r->stage = ST_MAIN;
        r->phase = PH_PREPARE;
        return;
    }
    const size_t nres = (size_t)(r->p.imax + 2) * (r->p.jmax + 2) * (r->ctx->kloc + 2);
    r->Q.assign(nres, 0.f);
    r->S.assign(nres, 0.f);
    const int rc = im.copy_out(s, r->Q.data(), r->S.data(), nullptr, nullptr, nullptr, nullptr);
    if (rc) {
        fail(sv, r, rc, r->ctx->err);
        return;
    }
    r->rel_std = rel_std_maxq(s.h_Qc, s.h_Sc, ncf);
    if (r->tol > 0) sv->calib[r->key] = std::make_pair(r->photmax, r->rel_std);
    s.state = 0;
    r->slot = nullptr;
    release_context(sv, r);
    r->stage = ST_DONE;
    r->t_done = now_s();
}

// Admit queued requests in arrival order while they fit.
void admit(rc_server *sv) {
    for (;;) {
        SrvReq *r = nullptr;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            if (sv->queue.empty() || (int)sv->running.size() >= sv->max_inflight) return;
            r = sv->queue.front();
            const size_t need = context_bytes(r->p, std::max(r->photmax, kPilotPhotmax));
            if (!has_idle_context(sv, r->key) && sv->hbm_in_use - idle_bytes(sv) + need > sv->budget &&
                !sv->running.empty())
                return;  // wait for running requests to give memory back
            sv->queue.pop_front();
        }
        r->t_admit = now_s();
        int rc = acquire_context(sv, r);
        if (!rc) {
            Impl<float> &im = *static_cast<Impl<float> *>(r->ctx->impl);
            r->slot = im.free_slot();
            r->slot->state = 3;
            rc = im.stage_host_field(*r->slot, r->T.data());
            if (rc) g_err = r->ctx->err;
        }
        std::lock_guard<std::mutex> lk(sv->mu);
        if (rc) {
            fail(sv, r, rc, g_err);
            r->published = true;
            sv->cv_done.notify_all();
            continue;
        }
        if (r->tol > 0) {
            auto it = sv->calib.find(r->key);
            if (it != sv->calib.end() && it->second.second > 0) {
                r->photmax = photmax_for(it->second.first, it->second.second, r->tol);
                r->stage = ST_MAIN;
            } else {
                r->photmax = kPilotPhotmax;
                r->stage = ST_PILOT;
            }
        } else {
            r->stage = ST_MAIN;
        }
        r->phase = PH_PREPARE;
        sv->running.push_back(r);
    }
}

bool quanta_in_flight(rc_server *sv) {
    for (int q = 0; q < rc_server::kNQ; ++q)
        if (sv->q_used[q] && cudaEventQuery(sv->mend[q]) != cudaSuccess) return true;
    return false;
}

void worker_loop(rc_server *sv) {
    cudaSetDevice(sv->device);
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            if (sv->stop) break;
        }
        admit(sv);
        // cancelled running requests: once no quantum or tally in flight
        // can still touch their slots, they end and give their contexts back
        {
            std::vector<SrvReq *> cancelled;
            {
                std::lock_guard<std::mutex> lk(sv->mu);
                for (SrvReq *r : sv->running)
                    if (r->cancel && r->stage < ST_DONE) cancelled.push_back(r);
            }
            if (!cancelled.empty()) {
                for (int q = 0; q < rc_server::kNQ; ++q) cudaStreamSynchronize(sv->qst[q]);
                cudaStreamSynchronize(sv->st);
                for (SrvReq *r : cancelled) {
                    if (r->slot) cudaStreamSynchronize(r->slot->st);
                    fail(sv, r, RC_E_CANCELLED, "request cancelled");
                }
            }
        }
        const int par = sv->q_par;
        // at most kNQ quanta in flight: this parity's previous quantum must
        // have finished before its stream and buffers take the next one
        if (sv->q_used[par]) cudaEventSynchronize(sv->mend[par]);
        if (sv->busy_since >= 0 && !quanta_in_flight(sv)) {
            std::lock_guard<std::mutex> lk(sv->mu);
            sv->busy_s += now_s() - sv->busy_since;
            sv->busy_since = -1.0;
        }
        // completed tallies
        bool progressed = false;
        for (SrvReq *r : sv->running)
            if (r->phase == PH_TALLY && r->stage < ST_DONE && cudaEventQuery(r->ev) == cudaSuccess) {
                finish_stage(sv, r);
                progressed = true;
            }
        bool prepare = false, tallying = false;
        int n_march = 0;
        for (SrvReq *r : sv->running) {
            if (r->stage >= ST_DONE) continue;
            prepare |= r->phase == PH_PREPARE;
            n_march += r->phase != PH_TALLY;
            tallying |= r->phase == PH_TALLY;
        }
        std::vector<SrvReq *> marching;
        if (n_march > 0) {
            cudaStream_t st = sv->qst[par];
            int rc = grow_quantum_buffers(sv, n_march);
            // the prelude follows the previous quantum's prelude
            if (!rc && sv->last_par >= 0) rc = cudaStreamWaitEvent(st, sv->pre_done[sv->last_par], 0) ? RC_E_CUDA : 0;
            if (rc) {
                for (SrvReq *r : sv->running)
                    if (r->stage < ST_DONE && r->phase != PH_TALLY) fail(sv, r, rc, sv->err);
            } else {
                if (prepare) {
                    // each starting request's field copy and set-up kernels
                    // form a chain of their own, forked round-robin over the
                    // side streams and joined before the quantum's march
                    std::vector<SrvReq *> starting;
                    for (SrvReq *r : sv->running)
                        if (r->stage < ST_DONE && r->phase == PH_PREPARE) starting.push_back(r);
                    const int ns = std::min<int>((int)starting.size(), rc_server::kSide);
                    bool forked = cudaEventRecord(sv->fork, st) == cudaSuccess;
                    for (int k = 0; k < ns && forked; ++k)
                        forked = cudaStreamWaitEvent(sv->side[k], sv->fork, 0) == cudaSuccess;
                    for (size_t i = 0; i < starting.size(); ++i) {
                        SrvReq *r = starting[i];
                        const int e = start_stage(sv, r, forked ? sv->side[i % ns] : st);
                        if (e) fail(sv, r, e, r->ctx ? r->ctx->err : g_err);
                    }
                    for (int k = 0; k < ns && forked; ++k) {
                        // a join that cannot be recorded is replaced by
                        // waiting for the side stream on the host
                        if (cudaEventRecord(sv->join[k], sv->side[k]) != cudaSuccess ||
                            cudaStreamWaitEvent(st, sv->join[k], 0) != cudaSuccess)
                            cudaStreamSynchronize(sv->side[k]);
                    }
                }
                for (SrvReq *r : sv->running)
                    if (r->stage < ST_DONE && r->phase == PH_MARCH) marching.push_back(r);
                if (!marching.empty()) {
                    if (sv->busy_since < 0) sv->busy_since = now_s();
                    rc = run_quantum(sv, marching, par);
                    if (!rc) {
                        sv->q_used[par] = true;
                        sv->last_par = par;
                        sv->q_par = (par + 1) % rc_server::kNQ;
                        rc = enqueue_tallies(sv, marching);
                    }
                    if (rc) {
                        for (int q = 0; q < rc_server::kNQ; ++q) cudaStreamSynchronize(sv->qst[q]);
                        cudaStreamSynchronize(sv->st);
                        for (SrvReq *r : marching) fail(sv, r, rc, sv->err);
                    }
                }
            }
        }
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            std::vector<SrvReq *> keep;
            for (SrvReq *r : sv->running) {
                if (r->stage >= ST_DONE) {
                    if (r->stage == ST_DONE) sv->solves_done += 1;
                    r->published = true;
                    progressed = true;
                } else {
                    keep.push_back(r);
                }
            }
            sv->running.swap(keep);
            if (progressed) sv->cv_done.notify_all();
        }
        if (marching.empty()) {
            if (tallying) {
                cudaStreamSynchronize(sv->st);
            } else if (!progressed) {
                std::unique_lock<std::mutex> lk(sv->mu);
                if (sv->running.empty())
                    sv->cv_work.wait_for(lk, std::chrono::milliseconds(5),
                                         [&] { return sv->stop || !sv->queue.empty(); });
            }
        }
    }
    for (int q = 0; q < rc_server::kNQ; ++q) cudaStreamSynchronize(sv->qst[q]);
    cudaStreamSynchronize(sv->st);
    // requests still queued or running end as failed
    std::lock_guard<std::mutex> lk(sv->mu);
    for (SrvReq *r : sv->running) {
        fail(sv, r, RC_E_STATE, "server destroyed");
        r->published = true;
    }
    sv->running.clear();
    for (SrvReq *r : sv->queue) {
        fail(sv, r, RC_E_STATE, "server destroyed");
        r->published = true;
    }
    sv->queue.clear();
    sv->cv_done.notify_all();
}

}  // namespace

extern "C" {

int rc_server_create(int device, double hbm_budget_bytes, int max_inflight, rc_server **out) {
    if (!out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    if (max_inflight < 1) return set_err(nullptr, RC_E_INVALID, "max_inflight must be >= 1");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_err(nullptr, RC_E_CUDA, cudaGetErrorString(e));
    auto *sv = new rc_server();
    sv->device = device;
    sv->budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : 150e9;
    sv->max_inflight = max_inflight;
    bool ok = cudaStreamCreateWithFlags(&sv->st, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; i < rc_server::kNQ && ok; ++i)
        ok = cudaStreamCreateWithFlags(&sv->qst[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaMalloc((void **)&sv->d_counter[i], sizeof(unsigned long long)) == cudaSuccess &&
             cudaEventCreateWithFlags(&sv->pre_done[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&sv->mend[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&sv->fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < rc_server::kSide && ok; ++i)
        ok = cudaStreamCreateWithFlags(&sv->side[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&sv->join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        rc_server_destroy(sv);
        return set_err(nullptr, RC_E_CUDA, "server stream/event creation failed");
    }
    sv->worker = std::thread(worker_loop, sv);
    *out = sv;
    return RC_OK;
}

int rc_server_set_scattering(rc_server *sv, int table_set, const rc_scattering *s) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    std::shared_ptr<ScatterSet> ss;
    if (s) {
        std::string err;
        if (scattering_check(*s, err)) return set_err(nullptr, RC_E_INVALID, err);
        ss = std::make_shared<ScatterSet>();
        ss->nB = s->nB;
        ss->nQ = s->nQ;
        ss->nA = s->nA;
        ss->ksca.assign(s->ksca, s->ksca + (size_t)s->nB * s->nQ);
        if (s->kabs) ss->kabs.assign(s->kabs, s->kabs + (size_t)s->nB * s->nQ);
        ss->theta.assign(s->theta, s->theta + s->nA);
        ss->cdf.assign(s->phase_cdf, s->phase_cdf + (size_t)s->nB * s->nA);
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (table_set < -1 || table_set >= (int)sv->tables.size())
        return set_err(nullptr, RC_E_INVALID, "unknown table set");
    if (ss) sv->scatter[table_set] = ss;
    else sv->scatter.erase(table_set);
    sv->scatter_gen[table_set] += 1;
    return RC_OK;
}

int rc_server_add_tables(rc_server *sv, const rc_tables *t, int *table_set) {
    if (!sv || !t || !table_set) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    auto ts = std::make_unique<TableSet>();
    ts->from_view(t);
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->tables.push_back(std::move(ts));
    *table_set = (int)sv->tables.size() - 1;
    return RC_OK;
}

int rc_server_submit(rc_server *sv, const rc_request *req, int64_t *id) {
    if (!sv || !req || !req->params || !req->T || !id) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::string err;
    if (params_validate(*req->params, err)) return set_err(nullptr, RC_E_INVALID, err);
    if (req->params->floatpoint) return set_err(nullptr, RC_E_INVALID, "the server runs FP32 march solves only");
    if (!(req->tolerance >= 0.f)) return set_err(nullptr, RC_E_INVALID, "tolerance must be >= 0");
    if (req->tolerance == 0.f && req->params->photmax < 1)
        return set_err(nullptr, RC_E_INVALID, "photmax must be >= 1 when no tolerance is given");
    const int kl = req->params->kmax / req->params->p_col;
    const int zs = req->zstart > 0 ? req->zstart : 1;
    if (zs + kl - 1 > req->params->kmax) return set_err(nullptr, RC_E_INVALID, "zstart out of range");
    auto r = std::make_unique<SrvReq>();
    r->p = *req->params;
    const size_t nf = (size_t)(r->p.imax + 2) * (r->p.jmax + 2) * (r->p.kmax + 2);
    r->T.assign(req->T, req->T + nf);
    r->zstart = zs;
    r->tol = req->tolerance;
    r->photmax = req->tolerance > 0 ? 0 : req->params->photmax;
    r->t_submit = now_s();
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!r->p.grey && (req->table_set < 0 || req->table_set >= (int)sv->tables.size()))
        return set_err(nullptr, RC_E_INVALID, "unknown table set");
    r->table_set = r->p.grey ? -1 : req->table_set;
    r->key = class_key(r->p, r->table_set);
    {
        // contexts are pooled per class and medium: a table set whose
        // particles change starts a new class
        auto it = sv->scatter.find(r->table_set);
        if (it != sv->scatter.end()) r->scatter = it->second;
        r->key += "/s" + std::to_string(sv->scatter_gen[r->table_set]);
    }
    if ((double)context_bytes(r->p, std::max(r->photmax, kPilotPhotmax)) > sv->budget)
        return set_err(nullptr, RC_E_NOMEM, "request larger than the HBM budget");
    if (sv->stop) return set_err(nullptr, RC_E_STATE, "server is shutting down");
    if (cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) != cudaSuccess)
        return set_err(nullptr, RC_E_CUDA, "event creation failed");
    r->id = sv->next_id++;
    *id = r->id;
    sv->queue.push_back(r.get());
    sv->reqs[r->id] = std::move(r);
    sv->cv_work.notify_all();
    return RC_OK;
}

int rc_server_wait(rc_server *sv, int64_t id, float *Q, float *sigma, rc_result_info *info) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return set_err(nullptr, RC_E_NOTFOUND, "unknown request id");
    SrvReq *r = it->second.get();
    sv->cv_done.wait(lk, [&] { return r->published; });
    if (Q && !r->Q.empty()) memcpy(Q, r->Q.data(), r->Q.size() * sizeof(float));
    if (sigma && !r->S.empty()) memcpy(sigma, r->S.data(), r->S.size() * sizeof(float));
    if (info) {
        info->t_submit = r->t_submit;
        info->t_admit = r->t_admit;
        info->t_done = r->t_done;
        info->photmax = r->photmax;
        info->rel_std_maxq = r->rel_std;
        info->status = r->status;
    }
    const int st = r->status;
    const std::string m = r->err;
    if (r->ev) cudaEventDestroy(r->ev);
    sv->reqs.erase(it);
    if (st) return set_err(nullptr, st, m);
    return RC_OK;
}

int rc_server_cancel(rc_server *sv, int64_t id) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return set_err(nullptr, RC_E_NOTFOUND, "unknown request id");
    SrvReq *r = it->second.get();
    if (r->published) return set_err(nullptr, RC_E_STATE, "request already finished");
    for (auto q = sv->queue.begin(); q != sv->queue.end(); ++q)
        if (*q == r) {
            // not admitted: nothing of it is on the device
            sv->queue.erase(q);
            r->status = RC_E_CANCELLED;
            r->err = "request cancelled";
            r->stage = ST_FAILED;
            r->t_done = now_s();
            r->published = true;
            sv->cv_done.notify_all();
            return RC_OK;
        }
    r->cancel = true;
    sv->cv_work.notify_all();
    return RC_OK;
}

int rc_server_set_quantum(rc_server *sv, long long tiles) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    if (tiles < 0) return set_err(nullptr, RC_E_INVALID, "quantum must be >= 1 tile (0: sized from the backlog)");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->quantum_tiles = tiles;
    return RC_OK;
}

int rc_server_set_policy(rc_server *sv, int policy) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    if (policy != RC_SCHED_FAIR && policy != RC_SCHED_SRPT) return set_err(nullptr, RC_E_INVALID, "unknown policy");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->policy = policy;
    return RC_OK;
}

int rc_server_quanta(rc_server *sv, long long *quanta) {
    if (!sv || !quanta) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    *quanta = sv->quanta;
    return RC_OK;
}

int rc_server_stats(rc_server *sv, double *solves, double *busy_s, double *hbm_in_use) {
    if (!sv) return set_err(nullptr, RC_E_INVALID, "NULL server");
    std::lock_guard<std::mutex> lk(sv->mu);
    if (solves) *solves = sv->solves_done;
    if (busy_s) *busy_s = sv->busy_s;
    if (hbm_in_use) *hbm_in_use = sv->hbm_in_use;
    return RC_OK;
}

int rc_server_destroy(rc_server *sv) {
    if (!sv) return RC_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->device);
    for (int i = 0; i < rc_server::kNQ; ++i)
        if (sv->qst[i]) cudaStreamSynchronize(sv->qst[i]);
    if (sv->st) cudaStreamSynchronize(sv->st);
    for (auto &pc : sv->pool) rc_destroy(pc.ctx);
    for (auto &kv : sv->reqs)
        if (kv.second->ev) cudaEventDestroy(kv.second->ev);
    for (int i = 0; i < rc_server::kNQ; ++i) {
        if (sv->d_solves[i]) cudaFree(sv->d_solves[i]);
        if (sv->d_tiles[i]) cudaFree(sv->d_tiles[i]);
        if (sv->d_base[i]) cudaFree(sv->d_base[i]);
        if (sv->h_tiles[i]) cudaFreeHost(sv->h_tiles[i]);
        if (sv->h_base[i]) cudaFreeHost(sv->h_base[i]);
        if (sv->d_counter[i]) cudaFree(sv->d_counter[i]);
        if (sv->pre_done[i]) cudaEventDestroy(sv->pre_done[i]);
        if (sv->mend[i]) cudaEventDestroy(sv->mend[i]);
        if (sv->qst[i]) cudaStreamDestroy(sv->qst[i]);
    }
    for (int i = 0; i < rc_server::kSide; ++i) {
        if (sv->side[i]) {
            cudaStreamSynchronize(sv->side[i]);
            cudaStreamDestroy(sv->side[i]);
        }
        if (sv->join[i]) cudaEventDestroy(sv->join[i]);
    }
    if (sv->fork) cudaEventDestroy(sv->fork);
    if (sv->st) cudaStreamDestroy(sv->st);
    delete sv;
    return RC_OK;
}

}  // extern "C"
