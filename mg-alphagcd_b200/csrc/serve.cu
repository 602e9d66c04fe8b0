// serve.cu -- the serving loop: continuous batching of Louvain jobs.
//
// Jobs are queued by any host thread.  `slots` worker threads each own a
// context (streams, workspaces) and a batch object that is reused from batch
// to batch, so a warm worker allocates and frees no device memory (cudaFree
// would wait for the whole device and stall the other workers).  A free
// worker takes the queued jobs in arrival order -- the head job and the ones
// behind it with the same kind of input and run options and a similar size
// (within 8x of the head job's memory estimate) -- until its share of the HBM
// budget (budget / slots, by a per-job upper-bound estimate) or the job cap is
// reached, and runs them as one batch; the workers' batches run on
// their own streams and overlap on the GPU.  A job is complete as soon as its
// own graph finishes inside the batch (batch_run's per-graph callback), not
// when the whole batch ends.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "handles.cuh"

using namespace mg;

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    bool csr = false;
    mg_gen_params gen{};
    // host CSR input (copied at submit)
    uint32_t n = 0;
    std::vector<uint64_t> off;
    std::vector<uint32_t> cols;
    std::vector<double> w;
    bool weighted = false;
    mg_run_opts opts{};
    bool keep = false;
    size_t bytes = 0;  // device memory estimate
    mg_job_info info{};
    std::vector<uint32_t> assignment;
};

// Upper bound of the device memory one graph adds to a batch: per vertex the
// run state (three assignment buffers, relabel, composition, k, sigma, sum_in,
// active lists, bins), per directed entry the union CSR, the generator's pairs
// and sort keys, and the coarsening keys of the first level.
size_t estimate_bytes(uint64_t n, uint64_t nnz) { return 160 * n + 64 * nnz + (1ull << 20); }

// largest size ratio (device-memory estimate) between two jobs of one batch
constexpr size_t kBatchSizeRatio = 8;

bool same_run(const mg_run_opts &a, const mg_run_opts &b) {
    return a.version == b.version && a.threshold == b.threshold && a.max_phases == b.max_phases &&
           a.precision == b.precision;
}

mg_run_opts default_run() {
    mg_run_opts o;
    o.version = 2;
    o.threshold = 1e-6;
    o.max_phases = 1000;
    o.precision = MG_PREC_FP64;
    o.verbose = 0;
    o.keep_levels = 0;
    return o;
}

}  // namespace

struct mg_server {
    mg_serve_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;
    std::vector<std::thread> workers;
    bool stopping = false;
    uint64_t next_id = 1, next_batch = 1;
    size_t share = 0, reserved = 0;
    uint64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, running = 0, batches = 0;
    std::vector<double> latencies;
    Clock::time_point t0 = Clock::now();
    std::string last_error;
    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void finish_job(mg_server *S, Job *j, int state, mg_status st) {
    j->info.state = state;
    j->info.status = st;
    j->info.finished_s = S->now();
    if (state == MG_JOB_DONE) {
        S->completed++;
        S->latencies.push_back(j->info.finished_s - j->info.submitted_s);
    } else if (state == MG_JOB_FAILED) {
        S->failed++;
    } else {
        S->cancelled++;
    }
}

// Pack host CSR jobs into one union and upload it.
void pack_csr(mg_batch *b, const std::vector<Job *> &take) {
    const uint32_t G = (uint32_t)take.size();
    std::vector<uint64_t> voff(G + 1, 0);
    for (uint32_t g = 0; g < G; g++) voff[g + 1] = voff[g] + take[g]->n;
    const uint64_t n = voff[G];
    std::vector<uint64_t> off(n + 1, 0);
    uint64_t nnz = 0;
    bool weighted = false;
    for (Job *j : take) {
        nnz += j->off.back();
        weighted |= j->weighted;
    }
    std::vector<uint32_t> cols(nnz);
    std::vector<double> w(weighted ? nnz : 0);
    uint64_t base = 0;
    for (uint32_t g = 0; g < G; g++) {
        const Job *j = take[g];
        for (uint32_t v = 0; v < j->n; v++) off[voff[g] + v + 1] = base + j->off[v + 1];
        const uint64_t e = j->off.back();
        std::copy(j->cols.begin(), j->cols.end(), cols.begin() + base);
        if (weighted) {
            if (j->weighted) std::copy(j->w.begin(), j->w.end(), w.begin() + base);
            else std::fill(w.begin() + base, w.begin() + base + e, 1.0);
        }
        base += e;
    }
    batch_from_host_csr(b, voff.data(), off.data(), cols.data(), weighted ? (const void *)w.data() : nullptr,
                        weighted ? MG_WEIGHT_F64 : MG_WEIGHT_UNIT);
}

void run_batch(mg_server *S, mg_ctx *ctx, mg_batch *b, const std::vector<Job *> &take) {
    b->graphs = (uint32_t)take.size();
    mg_batch_result res;
    GraphDoneFn done = [&](uint32_t g, const mg_batch_graph_summary &sum, const uint32_t *a) {
        Job *j = take[g];
        std::vector<uint32_t> kept;
        if (j->keep) kept.assign(a, a + sum.n);
        std::lock_guard<std::mutex> lk(S->mu);
        if (j->info.state != MG_JOB_RUNNING) return;
        j->info.graph = sum;
        j->assignment.swap(kept);
        finish_job(S, j, MG_JOB_DONE, MG_OK);
        S->running--;
        S->cv_done.notify_all();
    };
    mg_status st = MG_OK;
    std::string msg;
    try {
        MG_CUDA(cudaSetDevice(ctx->device));
        if (take[0]->csr) {
            pack_csr(b, take);
        } else {
            std::vector<mg_gen_params> gp;
            gp.reserve(take.size());
            for (Job *j : take) gp.push_back(j->gen);
            batch_generate(b, gp.data());
        }
        batch_run(b, take[0]->opts, S->opts.batch_flags, res, &done);
    } catch (const Error &e) {
        st = e.status;
        msg = e.what();
    } catch (const std::bad_alloc &) {
        st = MG_ERR_OOM;
        msg = "host allocation failed";
    } catch (const std::exception &e) {
        st = MG_ERR_INVALID;
        msg = e.what();
    }
    if (st != MG_OK) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->last_error = msg;
        for (Job *j : take)
            if (j->info.state == MG_JOB_RUNNING) {
                finish_job(S, j, MG_JOB_FAILED, st);
                S->running--;
            }
        S->cv_done.notify_all();
    }
}

void worker_main(mg_server *S) {
    mg_ctx *ctx = nullptr;
    mg_opts o = {S->opts.device, 0, 0};
    if (mg_init(&ctx, &o) != MG_OK) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->last_error = std::string("worker context: ") + mg_last_error(nullptr);
        return;
    }
    std::unique_ptr<mg_batch> b(new mg_batch());
    b->ctx = ctx;
    b->u.ctx = ctx;
    while (true) {
        std::vector<Job *> take;
        size_t used = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stopping || !S->queue.empty(); });
            if (S->stopping) break;
            const Job *head = S->queue.front();
            while (!S->queue.empty() && take.size() < S->opts.max_batch_jobs) {
                Job *j = S->queue.front();
                if (j->csr != head->csr || !same_run(j->opts, head->opts) || used + j->bytes > S->share) break;
                // jobs of similar size only: a batch holds its slot until its
                // slowest graph is done, so a large job among small ones would
                // keep the slot (and its memory share) long after they finished
                if (!take.empty() && (j->bytes > kBatchSizeRatio * head->bytes ||
                                      head->bytes > kBatchSizeRatio * j->bytes))
                    break;
                used += j->bytes;
                take.push_back(j);
                S->queue.pop_front();
            }
            const uint64_t batch = S->next_batch++;
            const double t = S->now();
            for (Job *j : take) {
                j->info.state = MG_JOB_RUNNING;
                j->info.started_s = t;
                j->info.batch = batch;
                j->info.batch_jobs = (uint32_t)take.size();
            }
            S->reserved += used;
            S->running += take.size();
            S->batches++;
        }
        run_batch(S, ctx, b.get(), take);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->reserved -= used;
            // CSR inputs are no longer needed
            for (Job *j : take) {
                std::vector<uint64_t>().swap(j->off);
                std::vector<uint32_t>().swap(j->cols);
                std::vector<double>().swap(j->w);
            }
        }
    }
    b.reset();
    mg_destroy(ctx);
}

mg_status serve_fail(mg_server *S, mg_status st, const std::string &msg) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->last_error = msg;
    return st;
}

mg_status enqueue(mg_server *S, std::unique_ptr<Job> j, const mg_run_opts *opts, int keep, uint64_t *id,
                  uint64_t n, uint64_t nnz) {
    j->opts = opts ? *opts : default_run();
    if (j->opts.version < 0 || j->opts.version > 2) return serve_fail(S, MG_ERR_INVALID, "version must be 0, 1 or 2");
    if (j->opts.precision < 0 || j->opts.precision > 2) return serve_fail(S, MG_ERR_INVALID, "unknown precision");
    j->keep = keep != 0;
    j->bytes = estimate_bytes(n, nnz);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) {
        S->last_error = "server is stopping";
        return MG_ERR_CANCELLED;
    }
    if (j->bytes > S->share) {
        S->last_error = "job larger than one slot's share of the HBM budget";
        return MG_ERR_OOM;
    }
    j->id = S->next_id++;
    j->info.state = MG_JOB_QUEUED;
    j->info.submitted_s = S->now();
    *id = j->id;
    S->queue.push_back(j.get());
    S->jobs[j->id] = std::move(j);
    S->submitted++;
    S->cv_work.notify_one();
    return MG_OK;
}

Job *find_job(mg_server *S, uint64_t id) {
    auto it = S->jobs.find(id);
    return it == S->jobs.end() ? nullptr : it->second.get();
}

bool finished(const Job *j) { return j->info.state >= MG_JOB_DONE; }

}  // namespace

extern "C" {

mg_status mg_serve_start(const mg_serve_opts *opts, mg_server **out) {
    if (!out) return MG_ERR_INVALID;
    *out = nullptr;
    mg_serve_opts o;
    o.device = 0;
    o.slots = 4;
    o.hbm_budget_bytes = (size_t)150e9;
    o.max_batch_jobs = 4096;
    o.batch_flags = MG_BATCH_GRAPHS;
    if (opts) o = *opts;
    if (o.slots < 1 || o.slots > 64 || o.max_batch_jobs < 1 || o.hbm_budget_bytes == 0) {
        set_orphan_error("mg_serve_start: bad options");
        return MG_ERR_INVALID;
    }
    mg_server *S = new (std::nothrow) mg_server();
    if (!S) return MG_ERR_OOM;
    S->opts = o;
    S->share = o.hbm_budget_bytes / (size_t)o.slots;
    try {
        for (int i = 0; i < o.slots; i++) S->workers.emplace_back(worker_main, S);
    } catch (const std::exception &e) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stopping = true;
        }
        S->cv_work.notify_all();
        for (auto &t : S->workers) t.join();
        delete S;
        set_orphan_error(std::string("mg_serve_start: ") + e.what());
        return MG_ERR_INVALID;
    }
    *out = S;
    return MG_OK;
}

mg_status mg_serve_submit(mg_server *S, const mg_gen_params *job, const mg_run_opts *opts, int keep_assignment,
                          uint64_t *id) {
    if (!S || !job || !id) return MG_ERR_INVALID;
    std::unique_ptr<Job> j(new (std::nothrow) Job());
    if (!j) return MG_ERR_OOM;
    j->gen = *job;
    uint64_t n = 0, nnz = 0;
    if (job->kind == MG_GEN_SBM) {
        if (job->blocks < 1 || job->n < job->blocks || !(job->mean_degree >= 0) || !(job->intra_frac >= 0) ||
            job->intra_frac > 1)
            return serve_fail(S, MG_ERR_INVALID, "sbm: bad parameters");
        n = job->n;
        nnz = 2 * (uint64_t)(job->n * job->mean_degree / 2.0 + 2.0);
    } else if (job->kind == MG_GEN_RMAT) {
        if (job->scale < 1 || job->scale > 30 || job->edge_factor < 1)
            return serve_fail(S, MG_ERR_INVALID, "rmat: bad scale or edge factor");
        n = 1ull << job->scale;
        nnz = 2 * ((uint64_t)job->edge_factor << job->scale);
    } else {
        return serve_fail(S, MG_ERR_INVALID, "unknown generator kind");
    }
    return enqueue(S, std::move(j), opts, keep_assignment, id, n, nnz);
}

mg_status mg_serve_submit_csr(mg_server *S, uint32_t n, const uint64_t *offsets, const uint32_t *cols,
                              const void *weights, int weight_type, const mg_run_opts *opts, int keep_assignment,
                              uint64_t *id) {
    if (!S || !offsets || !id) return MG_ERR_INVALID;
    if (weight_type < MG_WEIGHT_UNIT || weight_type > MG_WEIGHT_F64) return serve_fail(S, MG_ERR_INVALID, "bad weight type");
    const uint64_t nnz = offsets[n];
    if (offsets[0] != 0) return serve_fail(S, MG_ERR_INVALID, "offsets[0] must be 0");
    if (nnz && !cols) return serve_fail(S, MG_ERR_INVALID, "cols is NULL");
    if (nnz && weight_type != MG_WEIGHT_UNIT && !weights) return serve_fail(S, MG_ERR_INVALID, "weights is NULL");
    std::unique_ptr<Job> j;
    try {
        j.reset(new Job());
        j->csr = true;
        j->n = n;
        j->off.assign(offsets, offsets + (size_t)n + 1);
        j->cols.assign(cols, cols + nnz);
        if (weight_type != MG_WEIGHT_UNIT) {
            j->weighted = true;
            j->w.resize(nnz);
            for (uint64_t e = 0; e < nnz; e++)
                j->w[e] = weight_type == MG_WEIGHT_F32 ? (double)((const float *)weights)[e]
                                                       : ((const double *)weights)[e];
        }
    } catch (const std::bad_alloc &) {
        return serve_fail(S, MG_ERR_OOM, "host allocation failed");
    }
    return enqueue(S, std::move(j), opts, keep_assignment, id, n, nnz);
}

mg_status mg_serve_poll(mg_server *S, uint64_t id, mg_job_info *info) {
    if (!S || !info) return MG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Job *j = find_job(S, id);
    if (!j) {
        S->last_error = "no such job";
        return MG_ERR_INVALID;
    }
    *info = j->info;
    return MG_OK;
}

mg_status mg_serve_wait(mg_server *S, uint64_t id, double timeout_s, mg_job_info *info) {
    if (!S) return MG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    Job *j = find_job(S, id);
    if (!j) {
        S->last_error = "no such job";
        return MG_ERR_INVALID;
    }
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s));
    if (!S->cv_done.wait_until(lk, deadline, [&] { return finished(j); })) {
        if (info) *info = j->info;
        return MG_ERR_TIMEOUT;
    }
    if (info) *info = j->info;
    return MG_OK;
}

mg_status mg_serve_assignment(mg_server *S, uint64_t id, uint32_t *out) {
    if (!S || !out) return MG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Job *j = find_job(S, id);
    if (!j || j->info.state != MG_JOB_DONE || !j->keep) {
        S->last_error = "no kept assignment for this job";
        return MG_ERR_INVALID;
    }
    if (!j->assignment.empty()) memcpy(out, j->assignment.data(), sizeof(uint32_t) * j->assignment.size());
    return MG_OK;
}

mg_status mg_serve_cancel(mg_server *S, uint64_t id) {
    if (!S) return MG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Job *j = find_job(S, id);
    if (!j) return MG_ERR_INVALID;
    if (j->info.state != MG_JOB_QUEUED) return MG_ERR_INVALID;
    S->queue.erase(std::remove(S->queue.begin(), S->queue.end(), j), S->queue.end());
    finish_job(S, j, MG_JOB_CANCELLED, MG_ERR_CANCELLED);
    S->cv_done.notify_all();
    return MG_OK;
}

mg_status mg_serve_release(mg_server *S, uint64_t id) {
    if (!S) return MG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    Job *j = find_job(S, id);
    if (!j || !finished(j)) return MG_ERR_INVALID;
    S->jobs.erase(id);
    return MG_OK;
}

mg_status mg_serve_stats(mg_server *S, mg_serve_counters *out) {
    if (!S || !out) return MG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    mg_serve_counters c{};
    c.submitted = S->submitted;
    c.completed = S->completed;
    c.failed = S->failed;
    c.cancelled = S->cancelled;
    c.queued = S->queue.size();
    c.running = S->running;
    c.batches = S->batches;
    c.elapsed_s = S->now();
    c.jobs_per_s = c.elapsed_s > 0 ? (double)S->completed / c.elapsed_s : 0;
    if (!S->latencies.empty()) {
        std::vector<double> l = S->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            // nearest rank
            size_t r = (size_t)std::ceil(p * (double)l.size());
            return l[r == 0 ? 0 : r - 1];
        };
        c.p50_latency_s = pct(0.50);
        c.p99_latency_s = pct(0.99);
        double sum = 0;
        for (double x : l) sum += x;
        c.mean_latency_s = sum / (double)l.size();
        c.max_latency_s = l.back();
    }
    c.budget_bytes = S->opts.hbm_budget_bytes;
    c.reserved_bytes = S->reserved;
    *out = c;
    return MG_OK;
}

const char *mg_serve_last_error(mg_server *S) {
    if (!S) return "";
    std::lock_guard<std::mutex> lk(S->mu);
    static thread_local std::string copy;
    copy = S->last_error;
    return copy.c_str();
}

mg_status mg_serve_stop(mg_server *S) {
    if (!S) return MG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        for (Job *j : S->queue) finish_job(S, j, MG_JOB_CANCELLED, MG_ERR_CANCELLED);
        S->queue.clear();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    for (auto &t : S->workers) t.join();
    delete S;
    return MG_OK;
}

}  // extern "C"
