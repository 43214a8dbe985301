// rc_solver.cu -- C ABI of solver contexts, batched solves in one
// persistent launch (optionally a CUDA graph), bundle traces, the launch
// autotuner and the allocation-free solve, behind radchan.h.  The context
// implementation is in rc_impl.cuh.
#include "rc_impl.cuh"

using namespace rc_detail;


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

int rc_tables_validate(const rc_tables *t, char *msg, size_t msglen) {
    if (!t) return set_err(nullptr, RC_E_INVALID, "NULL tables");
    TableSet ts;
    ts.from_view(t);
    std::string err;
    const int rc = tables_check(ts, err);
    if (msg && msglen) snprintf(msg, msglen, "%s", err.c_str());
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_tables_view(const rc_table_set *ts, rc_tables *view) {
    if (!ts || !view) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    ts->ts.view(view);
    return RC_OK;
}

void rc_tables_free(rc_table_set *ts) { delete ts; }

int rc_scattering_synthetic(const rc_scatter_spec *spec, rc_scatter_set **out) {
    if (!spec || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    auto *s = new rc_scatter_set();
    std::string err;
    const int rc = scattering_synthetic(*spec, s->s, err);
    if (rc) {
        delete s;
        return set_err(nullptr, rc, err);
    }
    *out = s;
    return RC_OK;
}

int rc_scattering_read_dir(const char *dir, int nB, int nQ, rc_scatter_set **out) {
    if (!dir || !out) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    auto *s = new rc_scatter_set();
    std::string err;
    const int rc = scattering_read_dir(dir, nB, nQ, s->s, err);
    if (rc) {
        delete s;
        return set_err(nullptr, rc, err);
    }
    *out = s;
    return RC_OK;
}

int rc_scattering_write_dir(const rc_scatter_set *s, const char *dir) {
    if (!s || !dir) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    std::string err;
    const int rc = scattering_write_dir(s->s, dir, err);
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_scattering_validate(const rc_scattering *s, char *msg, size_t msglen) {
    if (!s) return set_err(nullptr, RC_E_INVALID, "NULL particle tables");
    std::string err;
    const int rc = scattering_check(*s, err);
    if (msg && msglen) snprintf(msg, msglen, "%s", err.c_str());
    if (rc) return set_err(nullptr, rc, err);
    return RC_OK;
}

int rc_scattering_view(const rc_scatter_set *s, rc_scattering *view) {
    if (!s || !view) return set_err(nullptr, RC_E_INVALID, "NULL argument");
    s->s.view(view);
    return RC_OK;
}

void rc_scattering_free(rc_scatter_set *s) { delete s; }

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

int rc_set_scattering(rc_ctx *c, const rc_scattering *s) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.set_scattering(s); });
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

int rc_collect_device(rc_ctx *c, rc_ticket t, double *q64, double *var64, double *qw64, double *vw64) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.collect_device(t, q64, var64, qw64, vw64); });
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
    c->gen++;
    return RC_OK;
}

int rc_set_priority(rc_ctx *c, float threshold) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    if (!(threshold >= 0.f) || threshold > 1e9f)
        return set_err(&c->err, RC_E_INVALID, "threshold must be a path length in [0, 1e9] channel widths");
    c->prio_thr = threshold;
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

int rc_sample_bands(rc_ctx *c, rc_ticket t, int kind, int n, const float *u_band, const float *u_g, int *nb,
                    int *g) {
    if (!c || (n > 0 && (!u_band || !u_g || !nb || !g)))
        return set_err(c ? &c->err : nullptr, RC_E_INVALID, "NULL argument");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) { return im.sample_bands(t, kind, n, u_band, u_g, nb, g); });
}

int rc_destroy(rc_ctx *c) {
    if (!c) return RC_OK;
    cudaSetDevice(c->device);
    if (c->impl) {
        if (c->dbl) delete static_cast<Impl<double> *>(c->impl);
        else delete static_cast<Impl<float> *>(c->impl);
    }
    if (c->d_dns) cudaFree(c->d_dns);
    if (c->d_dns_n) cudaFree(c->d_dns_n);
    if (c->h_dns) cudaFreeHost(c->h_dns);
    delete c;
    return RC_OK;
}

int rc_get_params(const rc_ctx *c, rc_params *p, int *device) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    if (p) *p = c->p;
    if (device) *device = c->device;
    return RC_OK;
}

int rc_last_error(const rc_ctx *c, char *buf, size_t len) {
    const std::string &m = c ? c->err : g_err;
    if (buf && len) snprintf(buf, len, "%s", m.c_str());
    return RC_OK;
}

int rc_debug_fail_next(const char *site, int count) {
    static const char *const sites[] = {"field_copy", "march", "tally", "collect", "dns", "quantum"};
    if (!site || count < 0) return set_err(nullptr, RC_E_INVALID, "NULL site or negative count");
    bool known = false;
    for (const char *s : sites) known = known || strcmp(s, site) == 0;
    if (!known) return set_err(nullptr, RC_E_INVALID, std::string("unknown failure site ") + site);
    FailPoints &f = fail_points();
    std::lock_guard<std::mutex> lk(f.mu);
    auto it = f.left.find(site);
    const bool was = it != f.left.end();
    if (count == 0) {
        if (was) {
            f.left.erase(it);
            f.armed.fetch_sub(1);
        }
    } else {
        f.left[site] = count;
        if (!was) f.armed.fetch_add(1);
    }
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
        unsigned long long gen;  // the context's generation the captured graph was built with
    };
    std::vector<Member> m;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // end of the set-up of every member, end of the march (phase timing)
    cudaEvent_t e_setup = nullptr, e_march = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool built = false;
    void *d_solves = nullptr, *h_solves = nullptr;
    long long *d_tiles = nullptr, *h_tiles = nullptr;
    TallyOut *d_outs = nullptr, *h_outs = nullptr;
    unsigned long long *d_counter = nullptr;
    size_t cap = 0;
    // the members' float results gathered into one buffer and copied to
    // the host once per run (k_copy_segs + one cudaMemcpyAsync)
    CopySeg *d_segs = nullptr, *h_segs = nullptr;  // n field segments, then 4 n result segments
    float *d_pack = nullptr, *h_pack = nullptr;
    size_t pack_cap = 0;
    std::vector<size_t> pack_off;
    // members' set-up chains run side by side on kSideStreams streams (forked
    // from and joined back into st: parallel branches of the captured graph)
    static constexpr int kSideStreams = 16;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork = nullptr, join[kSideStreams] = {};
    std::string err;
};

namespace {

template <typename R>
int batch_reserve(rc_batch *b, size_t n) {
    std::string *err_ = &b->err;
    if (5 * n > 65535) return set_err(err_, RC_E_INVALID, "more than 13107 solves in one batch");
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
    if (b->d_segs) cudaFree(b->d_segs);
    if (b->h_segs) cudaFreeHost(b->h_segs);
    b->d_segs = b->h_segs = nullptr;
    RC_CK(cudaMalloc((void **)&b->d_segs, 5 * n * sizeof(CopySeg)));
    RC_CK(cudaHostAlloc((void **)&b->h_segs, 5 * n * sizeof(CopySeg), cudaHostAllocDefault));
    b->cap = n;
    return RC_OK;
}

// The packed-results buffer, sized by the members' problems (allocated
// before any capture).
template <typename R>
int batch_reserve_members(rc_batch *b) {
    std::string *err_ = &b->err;
    size_t floats = 0;
    b->pack_off.assign(b->m.size(), 0);
    for (size_t i = 0; i < b->m.size(); ++i) {
        Impl<R> &im = *static_cast<Impl<R> *>(b->m[i].ctx->impl);
        b->pack_off[i] = floats;
        floats += im.packed_floats();
    }
    if (floats > b->pack_cap) {
        if (b->d_pack) cudaFree(b->d_pack);
        if (b->h_pack) cudaFreeHost(b->h_pack);
        b->d_pack = b->h_pack = nullptr;
        b->pack_cap = 0;
        RC_CK(cudaMalloc((void **)&b->d_pack, floats * sizeof(float)));
        RC_CK(cudaHostAlloc((void **)&b->h_pack, floats * sizeof(float), cudaHostAllocDefault));
        b->pack_cap = floats;
    }
    return RC_OK;
}

// The whole batch on b->st: per member field copy + set-up, one march
// over every member's tiles, one tally launch, scalars back.
template <typename R>
int batch_enqueue(rc_batch *b, bool capturing) {
    std::string *err_ = &b->err;
    // phase events: inside a captured graph they become event-record nodes
    auto mark = [&](cudaEvent_t ev) {
        return capturing ? cudaEventRecordWithFlags(ev, b->st, cudaEventRecordExternal) : cudaEventRecord(ev, b->st);
    };
    const size_t n = b->m.size();
    int rc = batch_reserve<R>(b, n);
    if (rc) return rc;
    DSolve<R> *hs = static_cast<DSolve<R> *>(b->h_solves);
    int rpt_max = 1, block = 256, scat = 0;
    long long max_cells = 1;
    b->h_tiles[0] = 0;
    // host halves: descriptors, tile prefix, tally outputs of every member
    long long maxf = 1;
    for (size_t i = 0; i < n; ++i) {
        rc_ctx *c = b->m[i].ctx;
        Impl<R> &im = *static_cast<Impl<R> *>(c->impl);
        if (im.nA > 0) scat = 1;  // the scattering variant of the march serves every member
        Slot<R> &s = *static_cast<Slot<R> *>(b->m[i].slot);
        rc = im.prepare_host(s, b->m[i].zstart, c->rpt);
        if (rc) return set_err(err_, rc, c->err);
        hs[i] = *s.h_desc;
        b->h_outs[i] = *s.h_out;
        b->h_tiles[i + 1] = b->h_tiles[i] + s.h_desc->n_tiles;
        rpt_max = std::max(rpt_max, c->rpt);
        if (i == 0) block = c->block;
        max_cells = std::max(max_cells, im.tally_cells());
        b->h_segs[i] = CopySeg{s.h_T, s.d_T, (long long)im.field_floats()};
        maxf = std::max(maxf, b->h_segs[i].n);
    }
    // one copy each of the descriptors, tile prefix and tally outputs; every
    // member's field in one launch that reads the pinned staging directly
    RC_CK(cudaMemcpyAsync(b->d_solves, hs, n * sizeof(DSolve<R>), cudaMemcpyHostToDevice, b->st));
    RC_CK(cudaMemcpyAsync(b->d_tiles, b->h_tiles, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, b->st));
    RC_CK(cudaMemcpyAsync(b->d_outs, b->h_outs, n * sizeof(TallyOut), cudaMemcpyHostToDevice, b->st));
    RC_CK(cudaMemcpyAsync(b->d_segs, b->h_segs, n * sizeof(CopySeg), cudaMemcpyHostToDevice, b->st));
    k_copy_segs<<<dim3((unsigned)std::min<long long>((maxf + 255) / 256, 64), (unsigned)n), 256, 0, b->st>>>(b->d_segs);
    RC_CK(cudaGetLastError());
    // every member's set-up kernels, round-robin over the side streams:
    // independent chains that run side by side, patching the batch's
    // descriptors in place
    const int ns = (int)std::min<size_t>(n, (size_t)rc_batch::kSideStreams);
    RC_CK(cudaEventRecord(b->fork, b->st));
    for (int k = 0; k < ns; ++k) RC_CK(cudaStreamWaitEvent(b->side[k], b->fork, 0));
    int rc_members = RC_OK;
    for (size_t i = 0; i < n && !rc_members; ++i) {
        rc_ctx *c = b->m[i].ctx;
        Impl<R> &im = *static_cast<Impl<R> *>(c->impl);
        Slot<R> &s = *static_cast<Slot<R> *>(b->m[i].slot);
        rc = im.prepare_device(s, nullptr, true, static_cast<DSolve<R> *>(b->d_solves) + i, b->side[i % ns]);
        if (rc) rc_members = set_err(err_, rc, c->err);
    }
    for (int k = 0; k < ns; ++k) {
        RC_CK(cudaEventRecord(b->join[k], b->side[k]));
        RC_CK(cudaStreamWaitEvent(b->st, b->join[k], 0));
    }
    if (rc_members) return rc_members;
    Impl<R> &im0 = *static_cast<Impl<R> *>(b->m[0].ctx->impl);
    RC_CK(mark(b->e_setup));
    rc = im0.launch_march(static_cast<const DSolve<R> *>(b->d_solves), b->d_tiles, (int)n, b->h_tiles[n],
                          b->d_counter, block, rpt_max, b->st, 0, nullptr, scat);
    if (rc) return set_err(err_, rc, b->m[0].ctx->err);
    RC_CK(mark(b->e_march));
    rc = im0.launch_tally(static_cast<const DSolve<R> *>(b->d_solves), b->d_outs, (int)n, max_cells, b->st);
    if (rc) return set_err(err_, rc, b->m[0].ctx->err);
    // float results of every member into one buffer, one copy to the host
    long long maxn = 1;
    CopySeg *rs = b->h_segs + n;
    for (size_t i = 0; i < n; ++i) {
        Impl<R> &im = *static_cast<Impl<R> *>(b->m[i].ctx->impl);
        im.pack_segments(*static_cast<Slot<R> *>(b->m[i].slot), b->d_pack + b->pack_off[i], rs + 4 * i);
        for (int q = 0; q < 4; ++q) maxn = std::max(maxn, rs[4 * i + q].n);
    }
    size_t floats = 0;
    for (size_t i = 0; i < n; ++i)
        floats += static_cast<Impl<R> *>(b->m[i].ctx->impl)->packed_floats();
    RC_CK(cudaMemcpyAsync(b->d_segs + n, rs, 4 * n * sizeof(CopySeg), cudaMemcpyHostToDevice, b->st));
    {
        const int gx = (int)std::min<long long>((maxn + 255) / 256, 64);
        k_copy_segs<<<dim3(gx, (unsigned)(4 * n)), 256, 0, b->st>>>(b->d_segs + n);
        RC_CK(cudaGetLastError());
    }
    RC_CK(cudaMemcpyAsync(b->h_pack, b->d_pack, floats * sizeof(float), cudaMemcpyDeviceToHost, b->st));
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
                int *sort_bands, int *occupancy) {
    if (!c) return set_err(nullptr, RC_E_INVALID, "NULL context");
    cudaSetDevice(c->device);
    return with_impl(c, [&](auto &im) {
        return im.autotune(T, zstart, pilot_photmax, rays_per_thread, block_threads, sort_bands, occupancy);
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
    if ((e = cudaEventCreate(&b->e_setup)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&b->e_march)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    for (int k = 0; k < rc_batch::kSideStreams; ++k) {
        if ((e = cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
        if ((e = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    }
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
        mm.gen = c->gen;
        b->m.push_back(mm);
        return RC_OK;
    });
    if (rc) return set_err(&b->err, rc, c->err);
    b->dbl = c->dbl;
    b->built = false;
    return RC_OK;
}

int rc_batch_run(rc_batch *b) {
    Range nv("rc_batch_run");
    if (!b) return set_err(nullptr, RC_E_INVALID, "NULL batch");
    if (b->m.empty()) return set_err(&b->err, RC_E_STATE, "empty batch");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    // the previous run reads the pinned descriptors and segment lists this
    // run rewrites: it finishes first
    RC_CK(cudaStreamSynchronize(b->st));
    // a member whose tables, particles or launch knobs changed since the
    // capture invalidates the graph (its descriptors and launch would be stale)
    for (auto &mm : b->m)
        if (mm.ctx->gen != mm.gen) {
            mm.gen = mm.ctx->gen;
            b->built = false;
        }
    int rc = b->dbl ? batch_ensure_scratch<double>(b) : batch_ensure_scratch<float>(b);
    if (rc) return rc;
    // all allocations happen before any stream capture
    rc = b->dbl ? batch_reserve<double>(b, b->m.size()) : batch_reserve<float>(b, b->m.size());
    if (rc) return rc;
    if (!b->built || !b->use_graph) {
        rc = b->dbl ? batch_reserve_members<double>(b) : batch_reserve_members<float>(b);
        if (rc) return rc;
    }
    if (!b->use_graph) {
        RC_CK(cudaEventRecord(b->e0, b->st));
        rc = b->dbl ? batch_enqueue<double>(b, false) : batch_enqueue<float>(b, false);
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
        rc = b->dbl ? batch_enqueue<double>(b, true) : batch_enqueue<float>(b, true);
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
    Range nv("rc_batch_wait");
    if (!b) return set_err(nullptr, RC_E_INVALID, "NULL batch");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    RC_CK(cudaEventSynchronize(b->e1));
    if (ms_device) RC_CK(cudaEventElapsedTime(ms_device, b->e0, b->e1));
    return RC_OK;
}

int rc_batch_phases(rc_batch *b, float *ms_setup, float *ms_march, float *ms_tally) {
    if (!b) return set_err(nullptr, RC_E_INVALID, "NULL batch");
    cudaSetDevice(b->device);
    std::string *err_ = &b->err;
    RC_CK(cudaEventSynchronize(b->e1));
    if (ms_setup) RC_CK(cudaEventElapsedTime(ms_setup, b->e0, b->e_setup));
    if (ms_march) RC_CK(cudaEventElapsedTime(ms_march, b->e_setup, b->e_march));
    if (ms_tally) RC_CK(cudaEventElapsedTime(ms_tally, b->e_march, b->e1));
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
    if (!q64 && !var64 && !qw64 && !vw64 && b->h_pack) {
        // float results only: from the copy every run makes of all members
        const float *pk = b->h_pack + b->pack_off[index];
        if (c->dbl) rc = static_cast<Impl<double> *>(c->impl)->collect_packed(*static_cast<Slot<double> *>(slot), pk,
                                                                             Q, sigma);
        else rc = static_cast<Impl<float> *>(c->impl)->collect_packed(*static_cast<Slot<float> *>(slot), pk, Q,
                                                                     sigma);
        if (rc) return set_err(&b->err, rc, c->err);
        return RC_OK;
    }
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
    if (b->d_segs) cudaFree(b->d_segs);
    if (b->h_segs) cudaFreeHost(b->h_segs);
    if (b->d_pack) cudaFree(b->d_pack);
    if (b->h_pack) cudaFreeHost(b->h_pack);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->e_setup) cudaEventDestroy(b->e_setup);
    if (b->e_march) cudaEventDestroy(b->e_march);
    if (b->fork) cudaEventDestroy(b->fork);
    for (int k = 0; k < rc_batch::kSideStreams; ++k) {
        if (b->side[k]) {
            cudaStreamSynchronize(b->side[k]);
            cudaStreamDestroy(b->side[k]);
        }
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
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
    // The tally writes only the walls whose flux is computed; the others read
    // 0, as the allocating entry points return them.
    const int nwalls = s.h_desc->nwalls;
    const size_t wall_bytes = 2 * (size_t)s.h_desc->nwc * sizeof(double);
    if (nwalls < 2 && qw64) RC_CK(cudaMemsetAsync(qw64, 0, wall_bytes, st));
    if (nwalls < 2 && vw64) RC_CK(cudaMemsetAsync(vw64, 0, wall_bytes, st));
    rc = im.launch_march(s.d_desc, s.d_tiles, 1, s.h_desc->n_tiles, s.d_counter, c->block, rpt, st);
    if (rc) return rc;
    rc = im.launch_tally(s.d_desc, s.d_out, 1, im.tally_cells(), st);
    if (rc) return rc;
    RC_CK(cudaMemcpyAsync(s.h_sc, s.d_sc, sizeof(DScalars), cudaMemcpyDeviceToHost, st));
    RC_CK(cudaStreamSynchronize(st));
    // No ticket exists to read rc_solve_info from, so the status word of the
    // solve travels in the return code and the message.  The outputs are
    // written in every case below.
    const int status = s.h_sc->status;
    if (status & 2) return set_err(err_, RC_E_RANGE, "temperature field contains non-finite values (status bit 1)");
    if (status & 8)
        return set_err(err_, RC_E_RANGE,
                       "an index was out of bounds in the march (status bit 3, bounds-checked build), first at site " +
                           std::to_string(s.h_sc->bad_site));
    if (status & 1)
        return set_err(err_, RC_E_RANGE,
                       "temperature outside the table range (status bit 0): results written with the end rows of "
                       "the tables (clamped)");
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
