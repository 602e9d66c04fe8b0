// ref_harness.cu -- drives the MG-alphaGCD reference's own code (built from
// its sources by oracle/build_ref.sh with the single-PE shim in
// oracle/ref_shim/) to produce golden vectors.  Test infrastructure only.
//
// Commands (all graphs are read through the reference's own .mtx loader,
// src/mmio/mmio_wrapper.cu:297):
//   load    <g.mtx> <out.bin>                       CSR as loaded (host only)
//   bins    <g.mtx> <out.bin>                       BIN::bin_create x3 (src/bin/BIN.cu:468-575)
//   move    <g.mtx> <C.bin> <sigma.bin> <k.bin> <up> <version> <out.bin>
//           one calculate_eicj_and_move_vertex_bin sweep
//           (src/louvain/louvain.cu:1032, src/louvain/louvain_gl.cu:1018)
//   coarsen <g.mtx> <C.bin> <out.bin>               coarsen_graph_mg::coarsen_graph
//           (src/coarsen_graph/coarsen_graph_mg.cu:2054)
//   louvain <g.mtx> <version>                       louvain*::run, prints the reference's table
//
// Binary layouts (little endian): see write_* below.
#include "common.h"
#include "graph/host_graph.h"
#include "graph/gpu_graph.cuh"
#include "bin/BIN.cuh"
#include "louvain/louvain.cuh"
#include "louvain/louvain_gl.cuh"
#include "louvain/louvain_baseline.cuh"
#include "coarsen_graph/coarsen_graph_mg.cuh"
#include "partition/edge_partition.cuh"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace louvain {
void calculate_eicj_and_move_vertex_bin(vertex_t, vertex_t, vertex_t *, edge_t *, weight_t *, weight_t *,
                                        vertex_t *, vertex_t *, vertex_t *, weight_t *, weight_t, int, int,
                                        bool, BIN *, cudaStream_t *, vertex_t, cudaStream_t);
}
namespace louvain_gl {
void calculate_eicj_and_move_vertex_bin(vertex_t, vertex_t, vertex_t *, edge_t *, weight_t *, weight_t *,
                                        vertex_t *, vertex_t *, vertex_t *, weight_t *, weight_t, int, int,
                                        bool, BIN *, cudaStream_t *, vertex_t, cudaStream_t);
}

static void die(const char *m) {
    fprintf(stderr, "ref_harness: %s\n", m);
    exit(2);
}

static void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
        exit(3);
    }
}

template <typename T>
static std::vector<T> read_vec(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) die("cannot open input vector");
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<T> v(sz / sizeof(T));
    if (!v.empty() && fread(v.data(), sizeof(T), v.size(), f) != v.size()) die("short read");
    fclose(f);
    return v;
}

// graph: u32 n, u32 nnz, u32 offsets[n+1], u32 cols[nnz], f64 weights[nnz]
static void write_graph(FILE *f, uint32_t n, uint32_t nnz, const uint32_t *off, const uint32_t *cols,
                        const double *w) {
    fwrite(&n, 4, 1, f);
    fwrite(&nnz, 4, 1, f);
    fwrite(off, 4, (size_t)n + 1, f);
    fwrite(cols, 4, nnz, f);
    fwrite(w, 8, nnz, f);
}

struct Loaded {
    HostGraph *host = nullptr;
    GpuGraph *gpu = nullptr;
};

static Loaded load_to_gpu(const char *path) {
    Loaded L;
    L.host = new HostGraph(const_cast<char *>(path), 0);
    L.host->compute_total_edge_weight();
    L.gpu = new GpuGraph(1, L.host);
    edge_partition::partitioner(L.host, L.gpu, 1, 0);
    ck(cudaDeviceSynchronize(), "partitioner");
    return L;
}

static int cmd_load(int argc, char **argv) {
    if (argc < 4) die("load <g.mtx> <out>");
    HostGraph h(argv[2], 0);
    FILE *f = fopen(argv[3], "wb");
    write_graph(f, h.get_total_vertices_(), h.get_total_edge_(), h.get_host_offset_(), h.get_host_edge_(),
                h.get_host_edge_weight_());
    fclose(f);
    return 0;
}

// bins: for each scheme s in {0 (10 bins), 1 (11 bins), 2 (9 bins)}:
//   u32 nbins, u32 sizes[nbins], u32 offsets[nbins], u32 max_degree, u32 n, u32 perm[n]
static int cmd_bins(int argc, char **argv) {
    if (argc < 4) die("bins <g.mtx> <out>");
    Loaded L = load_to_gpu(argv[2]);
    vertex_t n = L.gpu->get_local_vertices_();
    vertex_t *off = L.gpu->get_private_device_offset_();
    cudaStream_t s;
    ck(cudaStreamCreate(&s), "stream");
    FILE *f = fopen(argv[3], "wb");
    const int nb[3] = {BIN_NUM, BIN_NUM_COARSEN_GRAPH, BIN_NUM_COARSEN_GRAPH_NUMERIC};
    for (int scheme = 0; scheme < 3; scheme++) {
        BIN b(nb[scheme], n);
        if (scheme == 0) b.bin_create(off, n);
        else if (scheme == 1) b.bin_create(off, 0, n, s, 0);
        else b.bin_create(off, n, s, 0);
        ck(cudaDeviceSynchronize(), "bin_create");
        std::vector<uint32_t> perm(n);
        ck(cudaMemcpy(perm.data(), b.device_bin_permutation, 4ull * n, cudaMemcpyDeviceToHost), "perm");
        uint32_t k = nb[scheme];
        fwrite(&k, 4, 1, f);
        fwrite(b.bin_size, 4, k, f);
        fwrite(b.bin_offset, 4, k, f);
        fwrite(&b.max_degree, 4, 1, f);
        fwrite(&n, 4, 1, f);
        fwrite(perm.data(), 4, n, f);
    }
    fclose(f);
    return 0;
}

// move: u32 n, u32 C_new[n]
static int cmd_move(int argc, char **argv) {
    if (argc < 9) die("move <g.mtx> <C> <sigma> <k> <up> <version> <out>");
    Loaded L = load_to_gpu(argv[2]);
    auto C = read_vec<uint32_t>(argv[3]);
    auto sigma = read_vec<double>(argv[4]);
    auto k = read_vec<double>(argv[5]);
    bool up = atoi(argv[6]) != 0;
    int version = atoi(argv[7]);
    vertex_t n = L.gpu->get_local_vertices_();
    if (C.size() != n || sigma.size() != n || k.size() != n) die("vector sizes do not match the graph");
    ck(cudaMemcpy(L.gpu->get_shared_device_community_ids_(), C.data(), 4ull * n, cudaMemcpyHostToDevice), "C");
    ck(cudaMemcpy(L.gpu->get_shared_device_community_weight_(), sigma.data(), 8ull * n, cudaMemcpyHostToDevice), "sigma");
    ck(cudaMemcpy(L.gpu->get_private_device_vertex_weight_(), k.data(), 8ull * n, cudaMemcpyHostToDevice), "k");
    BIN *bins = new BIN(BIN_NUM, n);
    bins->bin_create(L.gpu->get_private_device_offset_(), n);
    cudaStream_t def, streams[STREAM_NUM];
    ck(cudaStreamCreate(&def), "stream");
    for (int i = 0; i < STREAM_NUM; i++) ck(cudaStreamCreate(&streams[i]), "stream");
    auto fn = version == 1 ? louvain_gl::calculate_eicj_and_move_vertex_bin : louvain::calculate_eicj_and_move_vertex_bin;
    fn(n, 0, L.gpu->get_private_device_offset_(), L.gpu->get_private_device_edge_(),
       L.gpu->get_private_device_edge_weight_(), L.gpu->get_private_device_vertex_weight_(),
       L.gpu->get_private_device_part_vertex_offset_(), L.gpu->get_shared_device_community_ids_new_(),
       L.gpu->get_shared_device_community_ids_(), L.gpu->get_shared_device_community_weight_(),
       L.host->get_mass_(), 0, 1, up, bins, streams, L.gpu->get_total_vertices_(), def);
    ck(cudaDeviceSynchronize(), "move");
    std::vector<uint32_t> out(n);
    ck(cudaMemcpy(out.data(), L.gpu->get_shared_device_community_ids_new_(), 4ull * n, cudaMemcpyDeviceToHost), "C_new");
    FILE *f = fopen(argv[8], "wb");
    fwrite(&n, 4, 1, f);
    fwrite(out.data(), 4, n, f);
    fclose(f);
    return 0;
}

// coarsen: graph layout of the next level
static int cmd_coarsen(int argc, char **argv) {
    if (argc < 5) die("coarsen <g.mtx> <C> <out>");
    Loaded L = load_to_gpu(argv[2]);
    auto C = read_vec<uint32_t>(argv[3]);
    vertex_t n = L.gpu->get_local_vertices_();
    if (C.size() != n) die("assignment size does not match the graph");
    ck(cudaMemcpy(L.gpu->get_shared_device_community_ids_(), C.data(), 4ull * n, cudaMemcpyHostToDevice), "C");
    cudaStream_t def, streams[STREAM_NUM];
    ck(cudaStreamCreate(&def), "stream");
    for (int i = 0; i < STREAM_NUM; i++) ck(cudaStreamCreate(&streams[i]), "stream");
    double t1 = 0, t2 = 0;
    coarsen_graph_mg::coarsen_graph(L.host, L.gpu, 0, 1, def, streams, t1, t2);
    ck(cudaDeviceSynchronize(), "coarsen");
    uint32_t n2 = L.gpu->get_local_vertices_();
    uint32_t e2 = L.gpu->get_local_edges_();
    std::vector<uint32_t> off(n2 + 1), cols(e2);
    std::vector<double> w(e2);
    ck(cudaMemcpy(off.data(), L.gpu->get_private_device_offset_(), 4ull * (n2 + 1), cudaMemcpyDeviceToHost), "off");
    ck(cudaMemcpy(cols.data(), L.gpu->get_private_device_edge_(), 4ull * e2, cudaMemcpyDeviceToHost), "cols");
    ck(cudaMemcpy(w.data(), L.gpu->get_private_device_edge_weight_(), 8ull * e2, cudaMemcpyDeviceToHost), "w");
    FILE *f = fopen(argv[4], "wb");
    write_graph(f, n2, e2, off.data(), cols.data(), w.data());
    fclose(f);
    return 0;
}

static int cmd_louvain(int argc, char **argv) {
    if (argc < 4) die("louvain <g.mtx> <version>");
    Loaded L = load_to_gpu(argv[2]);
    int version = atoi(argv[3]);
    if (version == 0) louvain_baseline::run(L.host, L.gpu, 1.0E-06, 500, 1000);
    else if (version == 1) louvain_gl::run(L.host, L.gpu, 1.0E-06, 500, 1000);
    else louvain::run(L.host, L.gpu, 1.0E-06, 500, 1000);
    ck(cudaDeviceSynchronize(), "louvain");
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 2) die("usage: ref_harness load|bins|move|coarsen|louvain ...");
    std::string c = argv[1];
    if (c == "load") return cmd_load(argc, argv);
    if (c == "bins") return cmd_bins(argc, argv);
    if (c == "move") return cmd_move(argc, argv);
    if (c == "coarsen") return cmd_coarsen(argc, argv);
    if (c == "louvain") return cmd_louvain(argc, argv);
    die("unknown command");
    return 2;
}
