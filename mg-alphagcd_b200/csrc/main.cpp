// main.cpp -- the MG_GCD command line, on top of libmgagcd.
//
// Flags follow src/main.cu:20-26 (parsed like get_argval, include/common.h:22-31:
// the value is the argument after the flag):
//   -path_of_graph <file.mtx>   input graph (Matrix Market, reference loader rules)
//   -threshold <double>         default 1e-6
//   -max_iter <int>             accepted and ignored, as in the reference
//   -max_phases <int>           default 1000
//   -version <0|1|2>            default 2 (0 behaves as 2 on one GPU)
//   -random_vertex_num <int>    size of the generated graph when no path is given (40)
//   -sparsity <double>          mean degree = sparsity * random_vertex_num (0.1)
// Additions of this engine:
//   -precision fp64|int64|fp32  gain arithmetic (default fp64 = reference)
//   -generator sbm|rmat         generated graph when no path is given (default sbm)
//   -scale <int> -edge_factor <int> -blocks <int> -seed <int>
//   -device <int>               CUDA device
//   -dump_assignment <file>     write "vertex community" lines (1-based like .mtx)
//   -csr_cache 0|1              read / write the binary CSR cache "<file>.mgcsr" (default 0)
// The reference's random graph (dense, directed, unseeded rand(),
// src/graph/host_graph.cpp:38-77) is replaced by the seeded generators.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "mgagcd.h"

template <typename T>
static T get_argval(char **begin, char **end, const std::string &arg, const T def) {
    T v = def;
    char **it = std::find(begin, end, arg);
    if (it != end && ++it != end) {
        std::istringstream in(*it);
        in >> v;
    }
    return v;
}

static int die(mg_ctx *ctx, mg_status st, const char *what) {
    fprintf(stderr, "MG_GCD: %s failed: %s (%s)\n", what, mg_status_string(st), mg_last_error(ctx));
    return 1;
}

int main(int argc, char **argv) {
    char **b = argv, **e = argv + argc;
    const std::string path = get_argval<std::string>(b, e, "-path_of_graph", "");
    const double threshold = get_argval<double>(b, e, "-threshold", 1.0e-06);
    (void)get_argval<int>(b, e, "-max_iter", 500);
    const int max_phases = get_argval<int>(b, e, "-max_phases", 1000);
    const int rvn = get_argval<int>(b, e, "-random_vertex_num", 40);
    const double sparsity = get_argval<double>(b, e, "-sparsity", 0.1);
    const int version = get_argval<int>(b, e, "-version", 2);
    const std::string prec = get_argval<std::string>(b, e, "-precision", "fp64");
    const std::string gen = get_argval<std::string>(b, e, "-generator", "sbm");
    const int scale = get_argval<int>(b, e, "-scale", 16);
    const int ef = get_argval<int>(b, e, "-edge_factor", 16);
    const int blocks = get_argval<int>(b, e, "-blocks", 4);
    const long long seed = get_argval<long long>(b, e, "-seed", 1);
    const int device = get_argval<int>(b, e, "-device", 0);
    const std::string dump = get_argval<std::string>(b, e, "-dump_assignment", "");
    const int csr_cache = get_argval<int>(b, e, "-csr_cache", 0);

    if (version < 0 || version > 2) {
        printf("the version is unsupported\n");
        return 0;
    }
    int precision = MG_PREC_FP64;
    if (prec == "int64") precision = MG_PREC_INT64;
    else if (prec == "fp32") precision = MG_PREC_FP32;
    else if (prec != "fp64") {
        fprintf(stderr, "MG_GCD: unknown -precision %s\n", prec.c_str());
        return 1;
    }

    mg_opts opts{device, 1, 0};
    mg_ctx *ctx = nullptr;
    mg_status st = mg_init(&ctx, &opts);
    if (st != MG_OK) return die(nullptr, st, "mg_init");
    mg_graph *g = nullptr;
    std::string name;
    if (!path.empty()) {
        printf("loading graph...\n");
        st = mg_graph_from_mtx_ex(ctx, path.c_str(), csr_cache ? MG_LOAD_CACHE_READ | MG_LOAD_CACHE_WRITE : 0, &g);
        name = path;
    } else if (gen == "rmat") {
        st = mg_graph_generate_rmat(ctx, scale, ef, 0.57, 0.19, 0.19, (uint64_t)seed, &g);
        name = "rmat-" + std::to_string(scale);
    } else {
        uint32_t n = (uint32_t)std::max(rvn, 1);
        uint32_t nb = (uint32_t)std::max(1, std::min<int>(blocks, (int)n));
        st = mg_graph_generate_sbm(ctx, n, nb, sparsity * n, 0.8, (uint64_t)seed, &g);
        name = "sbm";
    }
    if (st != MG_OK) {
        int r = die(ctx, st, "graph setup");
        mg_destroy(ctx);
        return r;
    }
    uint32_t n = 0;
    uint64_t nnz = 0;
    double mass = 0;
    int integral = 0;
    mg_graph_info(g, &n, &nnz, &mass, &integral);
    std::cout << std::setfill('-') << std::setw(3 * 25) << "" << std::setfill(' ') << std::endl;
    std::cout << std::setw(25) << "Input graph" << std::setw(25) << "Num. vertices (n)" << std::setw(25)
              << "Num. edges (M)" << std::endl;
    std::cout << std::setfill('-') << std::setw(3 * 25) << "" << std::setfill(' ') << std::endl;
    std::cout << std::setw(25) << name << std::setw(25) << n << std::setw(25) << nnz << std::endl;
    std::cout << std::setfill('-') << std::setw(3 * 25) << "" << std::setfill(' ') << std::endl;

    mg_run_opts ro{version, threshold, max_phases, precision, 1, 0};
    mg_result *res = nullptr;
    st = mg_louvain_run(g, &ro, &res);
    if (st != MG_OK) {
        int r = die(ctx, st, "mg_louvain_run");
        mg_graph_destroy(g);
        mg_destroy(ctx);
        return r;
    }
    mg_summary s{};
    mg_result_summary(res, &s);
    std::vector<uint32_t> levels(256);
    int nl = 0;
    mg_result_level_sizes(res, levels.data(), 256, &nl);
    printf("Modularity                  : %.9f\n", s.modularity);
    printf("Communities                 : %u\n", s.communities);
    printf("Levels (vertices per phase) :");
    for (int i = 0; i < nl && i < 256; i++) printf(" %u", levels[i]);
    printf("\n");
    if (!dump.empty()) {
        std::vector<uint32_t> a(n);
        mg_result_assignment(res, a.data());
        FILE *f = fopen(dump.c_str(), "w");
        if (f) {
            for (uint32_t v = 0; v < n; v++) fprintf(f, "%u %u\n", v + 1, a[v] + 1);
            fclose(f);
        }
    }
    mg_result_destroy(res);
    mg_graph_destroy(g);
    mg_destroy(ctx);
    return 0;
}
