// handles.cuh -- the opaque handles behind the C ABI (mg_ctx, mg_graph,
// mg_result) and the engine entry points the ABI calls.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "engine.cuh"

struct mg_ctx {
    int device = 0;
    int verbose = 0;
    size_t budget = 0;
    std::string last_error;
    cudaStream_t stream = nullptr;
    mg::MoveWorkspace mws;
    mg::CoarsenWorkspace cws;
    // Louvain run state (grow-only, reused across runs)
    mg::DBuf<uint32_t> C[3], Cd, assign, tmp32;
    mg::DBuf<double> k, sigma;
    mg::LevelGraph lv[2];
    mg::SweepAcc *h_acc = nullptr;  // pinned
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    ~mg_ctx();
};

struct mg_graph {
    mg_ctx *ctx = nullptr;
    uint32_t n = 0;
    uint64_t nnz = 0;
    mg::DBuf<uint32_t> off, col;
    mg::DBuf<float> w32;
    mg::DBuf<double> w64;
    int wk = mg::WK_UNIT;
    double mass = 0;
    int integral = 1;
    int sorted_rows = 0;  // every row strictly increasing (no repeated neighbour)
    int symmetric = 0;    // integral and symmetric as a multiset of entries (GraphView::symmetric)
    mg::GraphView view() const {
        mg::GraphView v;
        v.n = n;
        v.nnz = nnz;
        v.off = off.get();
        v.col = col.get();
        v.wk = wk;
        v.sorted_rows = sorted_rows != 0;
        v.symmetric = symmetric != 0;
        v.w = wk == mg::WK_F32 ? (const void *)w32.get() : wk == mg::WK_F64 ? (const void *)w64.get() : nullptr;
        return v;
    }
};

struct mg_result {
    uint32_t n0 = 0;
    mg_summary sum{};
    std::vector<uint32_t> assignment;
    std::vector<uint32_t> level_sizes;
    std::vector<double> trace;  // rows of 4
    std::vector<std::vector<uint32_t>> level_maps;  // dendrogram (keep_levels)
    // the graph every level worked on (keep_levels >= 2): offsets, columns,
    // weights as double
    struct LevelCsr {
        std::vector<uint32_t> off, col;
        std::vector<double> w;
    };
    std::vector<LevelCsr> level_csr;
};

namespace mg {
// per-graph sums of one batched sweep
struct GSum {
    unsigned long long sin_u, s2_u;
    double sin_f, s2_f;
};
// device-side control block of a batched run
struct BatchCtrl {
    int up;                     // direction of the next sweep
    int active;                 // graphs taking part in the next sweep
    unsigned long long sweeps;  // sweeps run
    unsigned long long edges;   // entries of the graphs that took part in them
    long long budget;           // sweeps left in this launch (CUDA-graph loop)
    unsigned long long active_vertices;  // vertices of the graphs active in the next sweep
    unsigned long long listed;  // vertices on the active lists (set by the host)
    unsigned long long pad[2];  // pad[0]: blocks done in the decision kernel
};
// Device state of a batch, resident between runs.
struct BatchWork {
    DBuf<uint32_t> gid, goff, goff_new, goff0, gword, gnnz, loops, Cf;
    // active lists: light-class entries (class order) and vertices (id order), each
    // with the graph of every entry; double-buffered for compaction
    DBuf<uint32_t> lperm[2], lpgid[2], lvert[2], lvgid[2], flags, pos;
    DBuf<double> sinv, curQ, gmass;
    DBuf<GainK> gk;
    DBuf<unsigned long long> iters;
    DBuf<GSum> sums;
    DBuf<BatchCtrl> ctrl;
    BatchCtrl *h_ctrl = nullptr;  // pinned
    // construction and run scratch, kept so that a batch object reused for
    // the next set of graphs allocates (and frees) nothing once warm
    DBuf<uint32_t> pu, pv, small;
    DBuf<uint64_t> off64, pbase;
    DBuf<unsigned char> gen;
    DBuf<int> bad;
    DBuf<uint8_t> alive;
    LevelGraph built;  // swapped with the union's buffers by the generator
    ~BatchWork();
};
}  // namespace mg

struct mg_batch {
    mg_ctx *ctx = nullptr;
    uint32_t graphs = 0;
    mg_graph u;                     // the packed union: rows and columns in union ids
    std::vector<uint32_t> voff;     // first vertex of each graph (graphs + 1)
    std::vector<uint64_t> eoff;     // first entry of each graph (graphs + 1)
    std::vector<double> mass;       // per graph
    std::vector<int> integral;      // per graph
    mg::BatchWork work;
};

struct mg_batch_result {
    uint32_t graphs = 0;
    mg_summary sum{};
    std::vector<mg_batch_graph_summary> per;
    std::vector<uint32_t> voff;        // first vertex of each graph
    std::vector<uint32_t> assignment;  // graph-local community of every packed vertex
};

namespace mg {

void ctx_prepare(mg_ctx *ctx);
// error text for entry points that run without a context (mg_last_error(NULL))
void set_orphan_error(const std::string &msg);
// graph construction
void graph_from_host_csr(mg_graph *g, uint32_t n, const uint64_t *offsets, const uint32_t *cols, const void *w,
                         int weight_type);
void graph_from_device_csr(mg_graph *g, uint32_t n, uint64_t nnz, const uint32_t *d_off, const uint32_t *d_cols,
                           const void *d_w, int weight_type);
void graph_from_level(mg_graph *g, LevelGraph &lv, int integral, double mass);
void graph_generate_rmat(mg_graph *g, int scale, int edge_factor, double a, double b, double c, uint64_t seed);
void graph_generate_sbm(mg_graph *g, uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
                        uint64_t seed);
void graph_generate_chunglu(mg_graph *g, uint32_t n, double exponent, double mean_degree, double max_degree,
                            int lognormal, uint64_t seed);
// Louvain
void louvain_run(mg_ctx *ctx, const mg_graph *g, const mg_run_opts &o, mg_result &res);
// batched form
void batch_generate(mg_batch *b, const mg_gen_params *params);
void batch_from_host_csr(mg_batch *b, const uint64_t *voff, const uint64_t *offsets, const uint32_t *cols,
                         const void *w, int weight_type);
// Called by batch_run, on its thread, as soon as graph g's result is final:
// its summary and its graph-local assignment (n_g entries).
using GraphDoneFn = std::function<void(uint32_t g, const mg_batch_graph_summary &sum, const uint32_t *assignment)>;
void batch_run(mg_batch *b, const mg_run_opts &o, int flags, mg_batch_result &res, const GraphDoneFn *done = nullptr);

}  // namespace mg
