// handles.cuh -- the opaque handles behind the C ABI (mg_ctx, mg_graph,
// mg_result) and the engine entry points the ABI calls.
#pragma once

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
    mg::GraphView view() const {
        mg::GraphView v;
        v.n = n;
        v.nnz = nnz;
        v.off = off.get();
        v.col = col.get();
        v.wk = wk;
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
};

namespace mg {

void ctx_prepare(mg_ctx *ctx);
// graph construction
void graph_from_host_csr(mg_graph *g, uint32_t n, const uint64_t *offsets, const uint32_t *cols, const void *w,
                         int weight_type);
void graph_from_device_csr(mg_graph *g, uint32_t n, uint64_t nnz, const uint32_t *d_off, const uint32_t *d_cols,
                           const void *d_w, int weight_type);
void graph_from_level(mg_graph *g, LevelGraph &lv, int integral, double mass);
void graph_generate_rmat(mg_graph *g, int scale, int edge_factor, double a, double b, double c, uint64_t seed);
void graph_generate_sbm(mg_graph *g, uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
                        uint64_t seed);
// host .mtx loader with the reference's rules; returns CSR in host vectors
mg_status load_mtx_host(const char *path, uint32_t &n, std::vector<uint64_t> &off, std::vector<uint32_t> &cols,
                        std::vector<double> &w, std::string &err);
// Louvain
void louvain_run(mg_ctx *ctx, const mg_graph *g, const mg_run_opts &o, mg_result &res);

}  // namespace mg
