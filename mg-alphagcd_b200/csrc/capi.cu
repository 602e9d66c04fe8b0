// capi.cu -- the extern "C" entry points declared in include/mgagcd.h.
// Every entry point catches engine errors and returns an mg_status; the
// message of the last failure is kept on the context.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "handles.cuh"
#include "host_csr.h"

using namespace mg;

namespace {

thread_local std::string g_orphan_error;

mg_status fail(mg_ctx *ctx, mg_status st, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    else g_orphan_error = msg;
    return st;
}

template <class F>
mg_status guarded(mg_ctx *ctx, F &&f) {
    try {
        if (ctx) MG_CUDA(cudaSetDevice(ctx->device));
        f();
        return MG_OK;
    } catch (const Error &e) {
        return fail(ctx, e.status, e.what());
    } catch (const std::bad_alloc &) {
        return fail(ctx, MG_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(ctx, MG_ERR_INVALID, e.what());
    }
}

__global__ void sigma_from_assignment_kernel(const uint32_t *C, const double *k, uint32_t n, double *sigma) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicAdd(sigma + C[v], k[v]);
}

// copy a host assignment to the device and check every id is < n
uint32_t *upload_assignment(mg_ctx *ctx, const uint32_t *C, uint32_t n, DBuf<uint32_t> &buf) {
    MG_CHECK(C != nullptr || n == 0, MG_ERR_INVALID, "assignment is NULL");
    for (uint32_t v = 0; v < n; v++) MG_CHECK(C[v] < n, MG_ERR_INVALID, "community id out of range");
    uint32_t *d = buf.ensure((size_t)n + 1);
    MG_CUDA(cudaMemcpyAsync(d, C, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    return d;
}

}  // namespace

mg_ctx::~mg_ctx() {
    if (h_acc) cudaFreeHost(h_acc);
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
}

namespace mg {
thread_local unsigned long long g_kernel_launches = 0;

static std::atomic<long long> g_alloc_fault_countdown{0};  // 0: disarmed

bool alloc_fault_due() {
    long long c = g_alloc_fault_countdown.load(std::memory_order_relaxed);
    while (c > 0) {
        if (g_alloc_fault_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    }
    return false;
}

// error text for entry points that run without a context (mg_last_error(NULL))
void set_orphan_error(const std::string &msg) { g_orphan_error = msg; }

void ctx_prepare(mg_ctx *ctx) {
    if (ctx->stream) return;
    MG_CUDA(cudaSetDevice(ctx->device));
    MG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    MG_CUDA(cudaMallocHost(&ctx->h_acc, sizeof(SweepAcc)));
    for (auto &e : ctx->ev) MG_CUDA(cudaEventCreate(&e));
    ctx->mws.init_streams();
}
}  // namespace mg

extern "C" {

const char *mg_status_string(mg_status s) {
    switch (s) {
        case MG_OK: return "ok";
        case MG_ERR_INVALID: return "invalid argument";
        case MG_ERR_CUDA: return "CUDA error";
        case MG_ERR_OOM: return "out of memory";
        case MG_ERR_IO: return "I/O error";
        case MG_ERR_FORMAT: return "malformed input";
        case MG_ERR_UNSUPPORTED: return "unsupported";
        case MG_ERR_TIMEOUT: return "device wait timed out";
        case MG_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char *mg_version(void) { return "mg-alphagcd-b200 0.1 (sm_100a)"; }

mg_status mg_init(mg_ctx **out, const mg_opts *opts) {
    if (!out) return fail(nullptr, MG_ERR_INVALID, "mg_init: out is NULL");
    *out = nullptr;
    mg_ctx *ctx = new (std::nothrow) mg_ctx();
    if (!ctx) return fail(nullptr, MG_ERR_OOM, "mg_init: host allocation failed");
    if (opts) {
        ctx->device = opts->device;
        ctx->verbose = opts->verbose;
        ctx->budget = opts->hbm_budget_bytes;
    }
    mg_status st = guarded(ctx, [&] {
        int count = 0;
        MG_CUDA(cudaGetDeviceCount(&count));
        MG_CHECK(ctx->device >= 0 && ctx->device < count, MG_ERR_INVALID, "mg_init: no such CUDA device");
        ctx_prepare(ctx);
    });
    if (st != MG_OK) {
        g_orphan_error = ctx->last_error;
        delete ctx;
        return st;
    }
    *out = ctx;
    return MG_OK;
}

mg_status mg_destroy(mg_ctx *ctx) {
    if (!ctx) return MG_ERR_INVALID;
    cudaSetDevice(ctx->device);
    delete ctx;
    return MG_OK;
}

const char *mg_last_error(const mg_ctx *ctx) { return ctx ? ctx->last_error.c_str() : g_orphan_error.c_str(); }

// ---- graphs -------------------------------------------------------------------

mg_status mg_graph_from_csr(mg_ctx *ctx, uint32_t n, const uint64_t *offsets, const uint32_t *cols,
                            const void *weights, int weight_type, mg_graph **out) {
    if (!ctx || !out) return fail(ctx, MG_ERR_INVALID, "mg_graph_from_csr: NULL argument");
    *out = nullptr;
    mg_graph *g = new (std::nothrow) mg_graph();
    if (!g) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    g->ctx = ctx;
    mg_status st = guarded(ctx, [&] { graph_from_host_csr(g, n, offsets, cols, weights, weight_type); });
    if (st != MG_OK) {
        delete g;
        return st;
    }
    *out = g;
    return MG_OK;
}

mg_status mg_graph_from_device_csr(mg_ctx *ctx, uint32_t n, uint64_t nnz, const uint32_t *d_offsets32,
                                   const uint32_t *d_cols, const void *d_weights, int weight_type, mg_graph **out) {
    if (!ctx || !out || !d_offsets32) return fail(ctx, MG_ERR_INVALID, "mg_graph_from_device_csr: NULL argument");
    *out = nullptr;
    mg_graph *g = new (std::nothrow) mg_graph();
    if (!g) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    g->ctx = ctx;
    mg_status st = guarded(ctx, [&] { graph_from_device_csr(g, n, nnz, d_offsets32, d_cols, d_weights, weight_type); });
    if (st != MG_OK) {
        delete g;
        return st;
    }
    *out = g;
    return MG_OK;
}

mg_status mg_graph_from_mtx(mg_ctx *ctx, const char *path, mg_graph **out) {
    return mg_graph_from_mtx_ex(ctx, path, 0, out);
}

mg_status mg_graph_from_mtx_ex(mg_ctx *ctx, const char *path, int flags, mg_graph **out) {
    if (!ctx || !out || !path) return fail(ctx, MG_ERR_INVALID, "mg_graph_from_mtx: NULL argument");
    *out = nullptr;
    mg_host_csr c;
    std::string err;
    mg_status st;
    try {
        st = load_mtx_csr(path, flags, c, err);
    } catch (const std::bad_alloc &) {
        return fail(ctx, MG_ERR_OOM, "host allocation failed while loading");
    }
    if (st != MG_OK) return fail(ctx, st, "mg_graph_from_mtx: " + err);
    return mg_graph_from_csr(ctx, c.n, c.off, c.cols, c.w, c.weighted ? MG_WEIGHT_F64 : MG_WEIGHT_UNIT, out);
}

mg_status mg_csr_from_mtx(const char *path, int flags, mg_host_csr **out) {
    if (!out || !path) return fail(nullptr, MG_ERR_INVALID, "mg_csr_from_mtx: NULL argument");
    *out = nullptr;
    mg_host_csr *c = new (std::nothrow) mg_host_csr();
    if (!c) return fail(nullptr, MG_ERR_OOM, "host allocation failed");
    std::string err;
    mg_status st;
    try {
        st = load_mtx_csr(path, flags, *c, err);
    } catch (const std::bad_alloc &) {
        st = MG_ERR_OOM;
        err = "host allocation failed while loading";
    }
    if (st != MG_OK) {
        delete c;
        return fail(nullptr, st, "mg_csr_from_mtx: " + err);
    }
    *out = c;
    return MG_OK;
}

mg_status mg_csr_info(const mg_host_csr *c, uint32_t *n, uint64_t *nnz, int *weighted, int *from_cache,
                      int *cache_written) {
    if (!c) return fail(nullptr, MG_ERR_INVALID, "mg_csr_info: NULL csr");
    if (n) *n = c->n;
    if (nnz) *nnz = c->nnz;
    if (weighted) *weighted = c->weighted;
    if (from_cache) *from_cache = c->from_cache;
    if (cache_written) *cache_written = c->cache_written;
    return MG_OK;
}

mg_status mg_csr_arrays(const mg_host_csr *c, const uint64_t **offsets, const uint32_t **cols,
                        const double **weights) {
    if (!c) return fail(nullptr, MG_ERR_INVALID, "mg_csr_arrays: NULL csr");
    if (offsets) *offsets = c->off;
    if (cols) *cols = c->cols;
    if (weights) *weights = c->w;
    return MG_OK;
}

void mg_csr_free(mg_host_csr *c) { delete c; }

mg_status mg_graph_generate_rmat(mg_ctx *ctx, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                                 mg_graph **out) {
    if (!ctx || !out) return fail(ctx, MG_ERR_INVALID, "mg_graph_generate_rmat: NULL argument");
    *out = nullptr;
    mg_graph *g = new (std::nothrow) mg_graph();
    if (!g) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    g->ctx = ctx;
    mg_status st = guarded(ctx, [&] { graph_generate_rmat(g, scale, edge_factor, a, b, c, seed); });
    if (st != MG_OK) {
        delete g;
        return st;
    }
    *out = g;
    return MG_OK;
}

mg_status mg_graph_generate_sbm(mg_ctx *ctx, uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
                                uint64_t seed, mg_graph **out) {
    if (!ctx || !out) return fail(ctx, MG_ERR_INVALID, "mg_graph_generate_sbm: NULL argument");
    *out = nullptr;
    mg_graph *g = new (std::nothrow) mg_graph();
    if (!g) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    g->ctx = ctx;
    mg_status st = guarded(ctx, [&] { graph_generate_sbm(g, n, blocks, mean_degree, intra_frac, seed); });
    if (st != MG_OK) {
        delete g;
        return st;
    }
    *out = g;
    return MG_OK;
}

mg_status mg_graph_generate_chunglu(mg_ctx *ctx, uint32_t n, double exponent, double mean_degree, double max_degree,
                                    int lognormal, uint64_t seed, mg_graph **out) {
    if (!ctx || !out) return fail(ctx, MG_ERR_INVALID, "mg_graph_generate_chunglu: NULL argument");
    *out = nullptr;
    mg_graph *g = new (std::nothrow) mg_graph();
    if (!g) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    g->ctx = ctx;
    mg_status st = guarded(ctx, [&] { graph_generate_chunglu(g, n, exponent, mean_degree, max_degree, lognormal, seed); });
    if (st != MG_OK) {
        delete g;
        return st;
    }
    *out = g;
    return MG_OK;
}

mg_status mg_graph_info(const mg_graph *g, uint32_t *n, uint64_t *nnz, double *mass, int *integral) {
    if (!g) return MG_ERR_INVALID;
    if (n) *n = g->n;
    if (nnz) *nnz = g->nnz;
    if (mass) *mass = g->mass;
    if (integral) *integral = g->integral;
    return MG_OK;
}

mg_status mg_graph_properties(const mg_graph *g, int *sorted_rows, int *symmetric) {
    if (!g) return MG_ERR_INVALID;
    if (sorted_rows) *sorted_rows = g->sorted_rows;
    if (symmetric) *symmetric = g->symmetric;
    return MG_OK;
}

mg_status mg_graph_copy_csr(const mg_graph *g, uint64_t *offsets, uint32_t *cols, double *weights) {
    if (!g) return MG_ERR_INVALID;
    mg_ctx *ctx = g->ctx;
    return guarded(ctx, [&] {
        cudaStream_t s = ctx->stream;
        if (offsets) {
            std::vector<uint32_t> o32((size_t)g->n + 1);
            MG_CUDA(cudaMemcpyAsync(o32.data(), g->off.get(), sizeof(uint32_t) * o32.size(), cudaMemcpyDeviceToHost, s));
            MG_CUDA(cudaStreamSynchronize(s));
            for (size_t i = 0; i < o32.size(); i++) offsets[i] = o32[i];
        }
        if (cols && g->nnz)
            MG_CUDA(cudaMemcpyAsync(cols, g->col.get(), sizeof(uint32_t) * g->nnz, cudaMemcpyDeviceToHost, s));
        if (weights && g->nnz) {
            if (g->wk == WK_F64) {
                MG_CUDA(cudaMemcpyAsync(weights, g->w64.get(), sizeof(double) * g->nnz, cudaMemcpyDeviceToHost, s));
            } else if (g->wk == WK_F32) {
                std::vector<float> w32(g->nnz);
                MG_CUDA(cudaMemcpyAsync(w32.data(), g->w32.get(), sizeof(float) * g->nnz, cudaMemcpyDeviceToHost, s));
                MG_CUDA(cudaStreamSynchronize(s));
                for (uint64_t e = 0; e < g->nnz; e++) weights[e] = w32[e];
            } else {
                for (uint64_t e = 0; e < g->nnz; e++) weights[e] = 1.0;
            }
        }
        MG_CUDA(cudaStreamSynchronize(s));
    });
}

mg_status mg_graph_destroy(mg_graph *g) {
    if (!g) return MG_ERR_INVALID;
    if (g->ctx) cudaSetDevice(g->ctx->device);
    delete g;
    return MG_OK;
}

// ---- stage hooks -----------------------------------------------------------------

mg_status mg_bins(mg_graph *g, int scheme, uint32_t *sizes, uint32_t *offsets, uint32_t *perm, uint32_t *max_degree) {
    if (!g) return MG_ERR_INVALID;
    mg_ctx *ctx = g->ctx;
    return guarded(ctx, [&] {
        ctx_prepare(ctx);
        MG_CHECK(scheme >= 0 && scheme <= 2, MG_ERR_INVALID, "bins: scheme must be 0, 1 or 2");
        Bins b;
        uint32_t *d_perm = ctx->tmp32.ensure((size_t)g->n + 1);
        compute_bins(scheme, g->n, g->off.get(), d_perm, b, ctx->stream, ctx->mws.prim);
        for (int i = 0; i < 11; i++) {
            if (sizes) sizes[i] = i < b.count ? b.size[i] : 0;
            if (offsets) offsets[i] = i < b.count ? b.offset[i] : 0;
        }
        if (max_degree) *max_degree = b.max_degree;
        if (perm && g->n) {
            MG_CUDA(cudaMemcpyAsync(perm, d_perm, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost, ctx->stream));
            MG_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    });
}

mg_status mg_bins_offsets(mg_ctx *ctx, int scheme, uint32_t n, const uint64_t *offsets, uint32_t *sizes,
                          uint32_t *bin_offsets, uint32_t *perm, uint32_t *max_degree) {
    if (!ctx || !offsets) return fail(ctx, MG_ERR_INVALID, "mg_bins_offsets: NULL argument");
    return guarded(ctx, [&] {
        ctx_prepare(ctx);
        MG_CHECK(scheme >= 0 && scheme <= 2, MG_ERR_INVALID, "bins: scheme must be 0, 1 or 2");
        std::vector<uint32_t> o32((size_t)n + 1);
        for (uint32_t i = 0; i <= n; i++) {
            MG_CHECK(offsets[i] < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "offsets must be below 2^32-1");
            MG_CHECK(i == 0 || offsets[i] >= offsets[i - 1], MG_ERR_INVALID, "offsets must be non-decreasing");
            o32[i] = (uint32_t)offsets[i];
        }
        DBuf<uint32_t> d_off;
        uint32_t *d = d_off.ensure((size_t)n + 1);
        MG_CUDA(cudaMemcpyAsync(d, o32.data(), sizeof(uint32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
        uint32_t *d_perm = ctx->tmp32.ensure((size_t)n + 1);
        Bins b;
        compute_bins(scheme, n, d, d_perm, b, ctx->stream, ctx->mws.prim);
        for (int i = 0; i < 11; i++) {
            if (sizes) sizes[i] = i < b.count ? b.size[i] : 0;
            if (bin_offsets) bin_offsets[i] = i < b.count ? b.offset[i] : 0;
        }
        if (max_degree) *max_degree = b.max_degree;
        if (perm && n) {
            MG_CUDA(cudaMemcpyAsync(perm, d_perm, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        }
        MG_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

mg_status mg_local_move(mg_graph *g, int version, int up, int precision, const uint32_t *C, const double *sigma,
                        const double *k, uint32_t *C_new, uint64_t *distinct) {
    if (!g || !C || !sigma || !k || !C_new) return fail(g ? g->ctx : nullptr, MG_ERR_INVALID, "mg_local_move: NULL argument");
    mg_ctx *ctx = g->ctx;
    return guarded(ctx, [&] {
        ctx_prepare(ctx);
        MG_CHECK(version >= 0 && version <= 2, MG_ERR_INVALID, "version must be 0, 1 or 2");
        MG_CHECK(precision >= 0 && precision <= 2, MG_ERR_INVALID, "unknown precision");
        cudaStream_t s = ctx->stream;
        const uint32_t n = g->n;
        uint32_t *dC = upload_assignment(ctx, C, n, ctx->C[0]);
        uint32_t *dN = ctx->C[1].ensure((size_t)n + 1);
        double *dk = ctx->k.ensure((size_t)n + 1);
        double *ds = ctx->sigma.ensure((size_t)n + 1);
        MG_CUDA(cudaMemcpyAsync(dk, k, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        MG_CUDA(cudaMemcpyAsync(ds, sigma, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if (n == 0) return;
        MoveLevel lvl;
        move_prepare_level(g->view(), lvl, ctx->mws, s);
        SweepParams sp;
        sp.version = version == 1 ? 1 : 2;
        sp.up = up ? 1 : 0;
        sp.precision = precision;
        sp.mass = g->mass;
        sp.integral = g->integral;
        sp.agg = 0;
        sp.split = sweep_split(ctx->mws, 0);
        sweep_reset_acc(ctx->mws, s);
        move_sweep(g->view(), lvl, ctx->mws, sp, dC, dN, dk, ds, s);
        MG_CUDA(cudaMemcpyAsync(C_new, dN, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaMemcpyAsync(ctx->h_acc, ctx->mws.acc.get(), sizeof(SweepAcc), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        MG_CHECK(ctx->h_acc->overflow == 0, MG_ERR_UNSUPPORTED, "local move: a cluster hash segment overflowed");
        if (distinct) *distinct = ctx->h_acc->distinct;
    });
}

mg_status mg_modularity(mg_graph *g, const uint32_t *C, double *q) {
    if (!g || !q) return MG_ERR_INVALID;
    mg_ctx *ctx = g->ctx;
    return guarded(ctx, [&] {
        ctx_prepare(ctx);
        cudaStream_t s = ctx->stream;
        const uint32_t n = g->n;
        if (n == 0 || g->mass <= 0) {
            *q = 0;
            return;
        }
        uint32_t *dC = upload_assignment(ctx, C, n, ctx->C[0]);
        uint32_t *dI = ctx->C[2].ensure((size_t)n + 1);
        uint32_t *dN = ctx->C[1].ensure((size_t)n + 1);
        double *dk = ctx->k.ensure((size_t)n + 1);
        double *ds = ctx->sigma.ensure((size_t)n + 1);
        level_init(g->view(), dk, ds, dI, s);
        MG_CUDA(cudaMemsetAsync(ds, 0, sizeof(double) * n, s));
        sigma_from_assignment_kernel<<<148 * 8, 256, 0, s>>>(dC, dk, n, ds);
        MG_LAUNCH_CHECK();
        MoveLevel lvl;
        move_prepare_level(g->view(), lvl, ctx->mws, s);
        SweepParams sp;
        sp.mass = g->mass;
        sp.integral = g->integral;
        sweep_reset_acc(ctx->mws, s);
        sigma_sumsq(ds, n, g->integral, ctx->mws, s);
        move_sweep(g->view(), lvl, ctx->mws, sp, dC, dN, dk, ds, s);  // sums the internal weight of C
        MG_CUDA(cudaMemcpyAsync(ctx->h_acc, ctx->mws.acc.get(), sizeof(SweepAcc), cudaMemcpyDeviceToHost, s));
        MG_CUDA(cudaStreamSynchronize(s));
        *q = modularity_from_acc(*ctx->h_acc, g->mass, g->integral);
    });
}

mg_status mg_coarsen(mg_graph *g, const uint32_t *C, uint32_t *C_dense, mg_graph **out) {
    if (!g || !out) return MG_ERR_INVALID;
    *out = nullptr;
    mg_ctx *ctx = g->ctx;
    mg_graph *ng = new (std::nothrow) mg_graph();
    if (!ng) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    ng->ctx = ctx;
    mg_status st = guarded(ctx, [&] {
        ctx_prepare(ctx);
        cudaStream_t s = ctx->stream;
        const uint32_t n = g->n;
        uint32_t *dC = upload_assignment(ctx, C, n, ctx->C[0]);
        uint32_t *dCd = ctx->Cd.ensure((size_t)n + 1);
        uint32_t nn = relabel_dense(dC, n, dCd, ctx->cws, s);
        LevelGraph lv;
        coarsen_level(g->view(), dCd, nn, g->integral, lv, ctx->cws, s, nullptr,
                      ctx->mws.coarsen_combine == MG_COMBINE_ON);
        if (C_dense && n) {
            MG_CUDA(cudaMemcpyAsync(C_dense, dCd, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
        }
        MG_CUDA(cudaStreamSynchronize(s));
        ng->n = lv.n;
        ng->nnz = lv.nnz;
        std::swap(ng->off.p, lv.off.p);
        std::swap(ng->off.cap, lv.off.cap);
        std::swap(ng->col.p, lv.col.p);
        std::swap(ng->col.cap, lv.col.cap);
        if (lv.wk == WK_U32) {
            level_weights_f64(lv.view(), ng->w64.ensure(lv.nnz + 1), s);
            MG_CUDA(cudaStreamSynchronize(s));
        } else {
            std::swap(ng->w64.p, lv.w.p);
            std::swap(ng->w64.cap, lv.w.cap);
        }
        ng->wk = WK_F64;
        ng->mass = g->mass;
        ng->integral = g->integral;
        ng->sorted_rows = 1;  // coarsened rows come out sorted by neighbour community
        ng->symmetric = lv.symmetric;
    });
    if (st != MG_OK) {
        delete ng;
        return st;
    }
    *out = ng;
    return MG_OK;
}

// ---- full Louvain ----------------------------------------------------------------

mg_status mg_louvain_run(mg_graph *g, const mg_run_opts *opts, mg_result **out) {
    if (!g || !out) return MG_ERR_INVALID;
    *out = nullptr;
    mg_ctx *ctx = g->ctx;
    mg_run_opts o;
    o.version = 2;
    o.threshold = 1e-6;
    o.max_phases = 1000;
    o.precision = MG_PREC_FP64;
    o.verbose = 0;
    o.keep_levels = 0;
    if (opts) o = *opts;
    if (o.version < 0 || o.version > 2) return fail(ctx, MG_ERR_INVALID, "version must be 0, 1 or 2");
    if (o.precision < 0 || o.precision > 2) return fail(ctx, MG_ERR_INVALID, "unknown precision");
    mg_result *r = new (std::nothrow) mg_result();
    if (!r) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    mg_status st = guarded(ctx, [&] { louvain_run(ctx, g, o, *r); });
    if (st != MG_OK) {
        delete r;
        return st;
    }
    *out = r;
    return MG_OK;
}

mg_status mg_result_summary(const mg_result *r, mg_summary *s) {
    if (!r || !s) return MG_ERR_INVALID;
    *s = r->sum;
    return MG_OK;
}

mg_status mg_result_assignment(const mg_result *r, uint32_t *out) {
    if (!r || !out) return MG_ERR_INVALID;
    if (r->n0) memcpy(out, r->assignment.data(), sizeof(uint32_t) * r->n0);
    return MG_OK;
}

mg_status mg_result_level_sizes(const mg_result *r, uint32_t *out, int max, int *count) {
    if (!r) return MG_ERR_INVALID;
    int c = (int)r->level_sizes.size();
    if (count) *count = c;
    if (out)
        for (int i = 0; i < c && i < max; i++) out[i] = r->level_sizes[i];
    return MG_OK;
}

mg_status mg_result_level_map(const mg_result *r, int level, uint32_t *out, uint32_t max, uint32_t *size) {
    if (!r || level < 0 || level >= (int)r->level_maps.size()) return MG_ERR_INVALID;
    const std::vector<uint32_t> &m = r->level_maps[(size_t)level];
    if (size) *size = (uint32_t)m.size();
    if (out) memcpy(out, m.data(), sizeof(uint32_t) * std::min<size_t>(m.size(), max));
    return MG_OK;
}

mg_status mg_result_level_csr(const mg_result *r, int level, uint32_t *n, uint64_t *nnz, uint64_t *offsets,
                              uint32_t *cols, double *weights) {
    if (!r || level < 0 || level >= (int)r->level_csr.size()) return MG_ERR_INVALID;
    const mg_result::LevelCsr &L = r->level_csr[(size_t)level];
    const uint32_t nn = (uint32_t)(L.off.size() - 1);
    if (n) *n = nn;
    if (nnz) *nnz = L.col.size();
    if (offsets)
        for (size_t i = 0; i < L.off.size(); i++) offsets[i] = L.off[i];
    if (cols && !L.col.empty()) memcpy(cols, L.col.data(), sizeof(uint32_t) * L.col.size());
    if (weights && !L.w.empty()) memcpy(weights, L.w.data(), sizeof(double) * L.w.size());
    return MG_OK;
}

mg_status mg_result_trace(const mg_result *r, double *rows4, int max_rows, int *count) {
    if (!r) return MG_ERR_INVALID;
    int c = (int)(r->trace.size() / 4);
    if (count) *count = c;
    if (rows4)
        for (int i = 0; i < c && i < max_rows; i++) memcpy(rows4 + 4 * i, r->trace.data() + 4 * i, 4 * sizeof(double));
    return MG_OK;
}

mg_status mg_result_destroy(mg_result *r) {
    if (!r) return MG_ERR_INVALID;
    delete r;
    return MG_OK;
}

// ---- autotuner ------------------------------------------------------------------

namespace {
std::string tune_text(const TuneTable &T) {
    std::string out;
    char line[160];
    for (const auto &kv : T.entries) {
        const uint32_t k = kv.first;
        snprintf(line, sizeof line, "%u %u %u %u %u %u %s %.3f\n", k & 7u, (k >> 3) & 3u, (k >> 5) & 3u,
                 (k >> 7) & 1u, (k >> 8) & 31u, k >> 13, shape_name(kv.second.shape), (double)kv.second.us);
        out += line;
    }
    return out;
}
}  // namespace

mg_status mg_tune_mode(mg_ctx *ctx, int mode) {
    if (!ctx) return MG_ERR_INVALID;
    if (mode < MG_TUNE_OFF || mode > MG_TUNE_ON) return fail(ctx, MG_ERR_INVALID, "mg_tune_mode: unknown mode");
    ctx->mws.tune.mode = mode;
    return MG_OK;
}

mg_status mg_test_fail_allocation(uint64_t nth, uint64_t *pending) {
    const long long before = g_alloc_fault_countdown.exchange((long long)nth);
    if (pending) *pending = before > 0 ? (uint64_t)before : 0;
    return MG_OK;
}

mg_status mg_sweep_options(mg_ctx *ctx, const mg_sweep_opts *opts) {
    if (!ctx) return MG_ERR_INVALID;
    const int fill = opts ? opts->cluster_fill : MG_FILL_AUTO;
    const int comb = opts ? opts->coarsen_combine : MG_COMBINE_AUTO;
    if (comb < MG_COMBINE_AUTO || comb > MG_COMBINE_ON)
        return fail(ctx, MG_ERR_INVALID, "mg_sweep_options: unknown coarsen_combine");
    if (opts && (opts->light_streams < 0 || opts->light_streams > MoveWorkspace::kStreams - 1))
        return fail(ctx, MG_ERR_INVALID, "mg_sweep_options: light_streams must be 0..7");
    const int gc = opts && opts->giant_class ? opts->giant_class : kFirstHeavyClass + kTiers - 1;
    if (fill < MG_FILL_AUTO || fill > MG_FILL_SPLIT) return fail(ctx, MG_ERR_INVALID, "mg_sweep_options: unknown fill");
    if (gc < kFirstHeavyClass || gc > kFirstHeavyClass + kTiers - 1)
        return fail(ctx, MG_ERR_INVALID, "mg_sweep_options: giant_class must be 0 or 13..18");
    ctx->mws.cluster_fill = fill;
    ctx->mws.giant_class = gc;
    ctx->mws.coarsen_combine = comb;
    ctx->mws.first_sweep_kernels = !(opts && opts->table_first_sweep);
    ctx->mws.light_streams =
        opts && opts->light_streams ? opts->light_streams : MoveWorkspace::kDefaultLightStreams;
    return MG_OK;
}

mg_status mg_tune_table(mg_ctx *ctx, char *buf, size_t cap, size_t *len) {
    if (!ctx) return MG_ERR_INVALID;
    return guarded(ctx, [&] {
        const std::string t = tune_text(ctx->mws.tune);
        if (len) *len = t.size();
        if (buf && cap) {
            const size_t n = t.size() < cap - 1 ? t.size() : cap - 1;
            memcpy(buf, t.data(), n);
            buf[n] = 0;
        }
    });
}

mg_status mg_tune_save(mg_ctx *ctx, const char *path) {
    if (!ctx || !path) return MG_ERR_INVALID;
    const std::string t = tune_text(ctx->mws.tune);
    FILE *f = fopen(path, "w");
    if (!f) return fail(ctx, MG_ERR_IO, std::string("mg_tune_save: cannot open ") + path);
    const bool ok = fwrite(t.data(), 1, t.size(), f) == t.size();
    fclose(f);
    return ok ? MG_OK : fail(ctx, MG_ERR_IO, "mg_tune_save: write failed");
}

mg_status mg_tune_load(mg_ctx *ctx, const char *path) {
    if (!ctx || !path) return MG_ERR_INVALID;
    FILE *f = fopen(path, "r");
    if (!f) return fail(ctx, MG_ERR_IO, std::string("mg_tune_load: cannot open ") + path);
    char line[256];
    std::map<uint32_t, TuneEntry> add;
    mg_status st = MG_OK;
    while (fgets(line, sizeof line, f)) {
        unsigned wk, prec, ver, bt, cls, bucket;
        char name[16];
        double us;
        if (sscanf(line, "%u %u %u %u %u %u %15s %lf", &wk, &prec, &ver, &bt, &cls, &bucket, name, &us) != 8 ||
            wk > 5 || prec > 2 || ver > 2 || bt > 1 || cls >= (unsigned)kLightClasses || bucket > 31) {
            st = MG_ERR_FORMAT;
            break;
        }
        int sh = -1;
        for (int i = 0; i < SH_COUNT; i++)
            if (strcmp(name, shape_name(i)) == 0) sh = i;
        if (sh < 0 || shape_capacity(sh) < (1u << cls)) {
            st = MG_ERR_FORMAT;
            break;
        }
        const uint32_t key = wk | prec << 3 | ver << 5 | bt << 7 | cls << 8 | bucket << 13;
        add[key] = TuneEntry{(uint8_t)sh, (float)us};
    }
    fclose(f);
    if (st != MG_OK) return fail(ctx, st, "mg_tune_load: malformed line");
    for (const auto &kv : add) ctx->mws.tune.entries[kv.first] = kv.second;
    return MG_OK;
}

// ---- batched form -------------------------------------------------------------

mg_status mg_batch_draw_sbm_params(uint32_t graphs, uint32_t n_min, uint32_t n_max, uint32_t blocks_min,
                                   uint32_t blocks_max, double deg_min, double deg_max, double intra_min,
                                   double intra_max, uint64_t seed, mg_sbm_params *out) {
    if (!out && graphs) return fail(nullptr, MG_ERR_INVALID, "mg_batch_draw_sbm_params: out is NULL");
    if (n_min < 1 || n_max < n_min || blocks_min < 1 || blocks_max < blocks_min || deg_max < deg_min ||
        intra_max < intra_min || intra_min < 0 || intra_max > 1)
        return fail(nullptr, MG_ERR_INVALID, "mg_batch_draw_sbm_params: bad ranges");
    const uint64_t key = rng_key(seed, 0x42415443ull);
    auto unif = [&](uint64_t ctr) { return (double)(rng_at(key, ctr) >> 11) * (1.0 / 9007199254740992.0); };
    const double l0 = std::log((double)n_min), l1 = std::log((double)n_max);
    for (uint32_t g = 0; g < graphs; g++) {
        mg_sbm_params &p = out[g];
        double nv = std::floor(std::exp(l0 + unif(5ull * g) * (l1 - l0)) + 0.5);
        nv = nv < n_min ? n_min : nv > n_max ? n_max : nv;
        p.n = (uint32_t)nv;
        const uint32_t bmax = blocks_max < p.n ? blocks_max : p.n;
        const uint32_t bmin = blocks_min < bmax ? blocks_min : bmax;
        p.blocks = bmin + (uint32_t)(unif(5ull * g + 1) * (double)(bmax - bmin + 1));
        if (p.blocks > bmax) p.blocks = bmax;
        p.mean_degree = deg_min + unif(5ull * g + 2) * (deg_max - deg_min);
        p.intra_frac = intra_min + unif(5ull * g + 3) * (intra_max - intra_min);
        p.seed = rng_at(key, 5ull * g + 4);
    }
    return MG_OK;
}

static mg_status batch_new(mg_ctx *ctx, uint32_t graphs, mg_batch **out, mg_batch **b) {
    if (!ctx || !out) return fail(ctx, MG_ERR_INVALID, "batch: NULL argument");
    *out = nullptr;
    if (graphs < 1) return fail(ctx, MG_ERR_INVALID, "batch: need at least one graph");
    *b = new (std::nothrow) mg_batch();
    if (!*b) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    (*b)->ctx = ctx;
    (*b)->u.ctx = ctx;
    (*b)->graphs = graphs;
    return MG_OK;
}

mg_status mg_batch_generate(mg_ctx *ctx, uint32_t graphs, const mg_gen_params *params, mg_batch **out) {
    mg_batch *b = nullptr;
    mg_status st = batch_new(ctx, graphs, out, &b);
    if (st != MG_OK) return st;
    st = guarded(ctx, [&] { batch_generate(b, params); });
    if (st != MG_OK) {
        delete b;
        return st;
    }
    *out = b;
    return MG_OK;
}

mg_status mg_batch_generate_sbm(mg_ctx *ctx, uint32_t graphs, const mg_sbm_params *params, mg_batch **out) {
    mg_batch *b = nullptr;
    mg_status st = batch_new(ctx, graphs, out, &b);
    if (st != MG_OK) return st;
    st = guarded(ctx, [&] {
        MG_CHECK(params != nullptr, MG_ERR_INVALID, "batch: params is NULL");
        std::vector<mg_gen_params> gp(graphs);
        for (uint32_t g = 0; g < graphs; g++) {
            gp[g] = mg_gen_params{};
            gp[g].kind = MG_GEN_SBM;
            gp[g].n = params[g].n;
            gp[g].blocks = params[g].blocks;
            gp[g].mean_degree = params[g].mean_degree;
            gp[g].intra_frac = params[g].intra_frac;
            gp[g].seed = params[g].seed;
        }
        batch_generate(b, gp.data());
    });
    if (st != MG_OK) {
        delete b;
        return st;
    }
    *out = b;
    return MG_OK;
}

mg_status mg_batch_from_csr(mg_ctx *ctx, uint32_t graphs, const uint64_t *vertex_offsets, const uint64_t *offsets,
                            const uint32_t *cols, const void *weights, int weight_type, mg_batch **out) {
    mg_batch *b = nullptr;
    mg_status st = batch_new(ctx, graphs, out, &b);
    if (st != MG_OK) return st;
    st = guarded(ctx, [&] { batch_from_host_csr(b, vertex_offsets, offsets, cols, weights, weight_type); });
    if (st != MG_OK) {
        delete b;
        return st;
    }
    *out = b;
    return MG_OK;
}

mg_status mg_batch_info(const mg_batch *b, uint32_t *graphs, uint64_t *n, uint64_t *nnz) {
    if (!b) return MG_ERR_INVALID;
    if (graphs) *graphs = b->graphs;
    if (n) *n = b->u.n;
    if (nnz) *nnz = b->u.nnz;
    return MG_OK;
}

mg_status mg_batch_graph_info(const mg_batch *b, uint32_t g, uint32_t *n, uint64_t *nnz, double *mass) {
    if (!b) return MG_ERR_INVALID;
    if (g >= b->graphs) return fail(b->ctx, MG_ERR_INVALID, "batch: graph index out of range");
    if (n) *n = b->voff[g + 1] - b->voff[g];
    if (nnz) *nnz = b->eoff[g + 1] - b->eoff[g];
    if (mass) *mass = b->mass[g];
    return MG_OK;
}

mg_status mg_batch_destroy(mg_batch *b) {
    if (!b) return MG_ERR_INVALID;
    cudaSetDevice(b->ctx->device);
    delete b;
    return MG_OK;
}

mg_status mg_batch_run(mg_batch *b, const mg_run_opts *opts, int flags, mg_batch_result **out) {
    if (!b || !out) return MG_ERR_INVALID;
    *out = nullptr;
    mg_ctx *ctx = b->ctx;
    mg_run_opts o;
    o.version = 2;
    o.threshold = 1e-6;
    o.max_phases = 1000;
    o.precision = MG_PREC_FP64;
    o.verbose = 0;
    o.keep_levels = 0;
    if (opts) o = *opts;
    if (o.version < 0 || o.version > 2) return fail(ctx, MG_ERR_INVALID, "version must be 0, 1 or 2");
    if (o.precision < 0 || o.precision > 2) return fail(ctx, MG_ERR_INVALID, "unknown precision");
    if (flags & ~MG_BATCH_GRAPHS) return fail(ctx, MG_ERR_INVALID, "unknown batch flags");
    mg_batch_result *r = new (std::nothrow) mg_batch_result();
    if (!r) return fail(ctx, MG_ERR_OOM, "host allocation failed");
    mg_status st = guarded(ctx, [&] { batch_run(b, o, flags, *r); });
    if (st != MG_OK) {
        delete r;
        return st;
    }
    *out = r;
    return MG_OK;
}

mg_status mg_batch_result_summary(const mg_batch_result *r, mg_summary *s) {
    if (!r || !s) return MG_ERR_INVALID;
    *s = r->sum;
    return MG_OK;
}

mg_status mg_batch_result_graph(const mg_batch_result *r, uint32_t g, mg_batch_graph_summary *out) {
    if (!r || !out || g >= r->graphs) return MG_ERR_INVALID;
    *out = r->per[g];
    return MG_OK;
}

mg_status mg_batch_result_assignment(const mg_batch_result *r, uint32_t g, uint32_t *out) {
    if (!r || !out || g >= r->graphs) return MG_ERR_INVALID;
    const uint32_t n = r->voff[g + 1] - r->voff[g];
    if (n) memcpy(out, r->assignment.data() + r->voff[g], sizeof(uint32_t) * n);
    return MG_OK;
}

mg_status mg_batch_result_destroy(mg_batch_result *r) {
    if (!r) return MG_ERR_INVALID;
    delete r;
    return MG_OK;
}

}  // extern "C"
