/*
 * oracle.h -- CPU restatement of the MG-alphaGCD Louvain hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; it is used by tests/, by __graft_entry__.smoke() as the
 * checker, and by bench.py's cpu_baseline / --impl reference leg.
 *
 * Every function restates one piece of the reference and cites the file:line
 * it follows (paths relative to the MG-alphaGCD source tree).  Pinning: the
 * loader is pinned against the reference's own loader compiled from its
 * sources (oracle/build_ref.sh -> oracle/_ref/), the hot-path stages against
 * fixtures produced by the reference's kernels (tests/golden/).
 *
 * Conventions: a graph is a CSR with n vertices, offsets[n+1] (uint64),
 * cols[nnz] (uint32) and weights[nnz] (double) or NULL for unit weights.
 * Functions return 0 on success, a negative code on error.
 */
#ifndef MG_ORACLE_H
#define MG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t n;
    uint64_t nnz;
    uint64_t *offsets;   /* n+1 */
    uint32_t *cols;      /* nnz */
    double *weights;     /* nnz or NULL (unit) */
} or_graph;

void or_free(void *p);
void or_graph_free(or_graph *g);
int or_set_threads(int nthreads);
int or_get_threads(void);

/* ---- loader: src/mmio/mmio_wrapper.cu:76-295 ---------------------------- */
int or_load_mtx(const char *path, or_graph *out);

/* ---- generators (seeded, integer-only RNG; identical to the CUDA ones) --- */
uint64_t or_mix64(uint64_t x);
int or_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                uint64_t seed, or_graph *out);
int or_gen_sbm(uint32_t n, uint32_t blocks, double mean_degree, double intra_frac,
               uint64_t seed, or_graph *out);
int or_gen_chunglu(uint32_t n, double exponent, double mean_degree, double max_degree,
                   int lognormal_weights, uint64_t seed, or_graph *out);
/* Build a symmetric deduplicated CSR (rows sorted) from undirected pairs.
 * Self-loops dropped.  weights (per pair) may be NULL. */
int or_csr_from_pairs(uint32_t n, uint64_t m, const uint32_t *u, const uint32_t *v,
                      const double *w, or_graph *out);

/* ---- degree binning: src/bin/BIN.cu:33-575 -------------------------------
 * scheme 0: local-move 10 bins on row lengths (BIN.cu:72-92)
 * scheme 1: coarsen-symbolic 11 bins (BIN.cu:159-181)
 * scheme 2: coarsen-numeric 9 bins (BIN.cu:248-266)
 * degree of item i = offsets[i+1]-offsets[i].  sizes/offsets have 11 slots.
 * perm lists items bin by bin, ascending id inside a bin. */
int or_bins(int scheme, uint32_t n, const uint64_t *offsets, uint32_t *sizes,
            uint32_t *bin_offsets, uint32_t *perm, uint32_t *max_degree);

/* ---- one local-move sweep: src/louvain/louvain.cu:404-1030 (version 2),
 *      src/louvain/louvain_gl.cu:504,578 (version 1).
 * mass = sum of all directed weights (host_graph.cpp:112-115). */
int or_local_move(const or_graph *g, int version, int up, const uint32_t *C,
                  const double *sigma_tot, const double *k, double mass,
                  uint32_t *C_new, uint64_t *distinct_pairs);

/* vertex weights k_i = row sums (louvain.cu:30-74) */
int or_vertex_weights(const or_graph *g, double *k);
double or_mass(const or_graph *g);
/* graph has integral weights whose total fits 2^53 */
int or_is_integral(const or_graph *g);

/* ---- modularity: src/louvain/louvain.cu:105-238 -------------------------
 * Q = sum_in/mass - sum_c sigma_c^2 / mass^2, sigma given explicitly. */
double or_modularity_sigma(const or_graph *g, const uint32_t *C, const double *sigma,
                           double mass, int integral);
/* FP64 modularity recomputed from an assignment alone (sigma from C). */
double or_modularity(const or_graph *g, const uint32_t *C);

/* ---- coarsening: src/coarsen_graph/coarsen_graph_mg.cu:1330-2240 ---------
 * Dense order-preserving relabel of C (written to C_dense, may alias C),
 * next-level CSR with rows sorted by neighbour community, self-loops kept. */
int or_coarsen(const or_graph *g, const uint32_t *C, uint32_t *C_dense, or_graph *out,
               uint64_t *upper_degree /* n_new+1 offsets of upper bounds, may be NULL */);

/* ---- full Louvain: src/louvain/louvain.cu:1401-1715 ----------------------
 * trace: per iteration record {phase, loop, Q, dQ} in doubles (4 per row),
 *        loop 0 rows are the phase-start modularity.  max_trace rows.
 * level_sizes: vertex count at the start of each phase (max_levels).
 * assignment: composed final community of each original vertex (dense ids). */
typedef struct {
    double modularity;
    int phases;             /* phases run */
    int levels;             /* entries in level_sizes */
    int iterations;         /* total local-move sweeps */
    int trace_rows;
    uint32_t communities;   /* final community count */
} or_result;

int or_louvain(const or_graph *g, int version, double threshold, int max_phases,
               uint32_t *assignment, double *trace, int max_trace,
               uint32_t *level_sizes, int max_levels, or_result *res);

/* bounded timing sample: run `iters` local-move sweeps (+sigma update) of
 * phase 0 and return seconds spent (for the CPU baseline). */
double or_time_phase0(const or_graph *g, int version, int iters, uint64_t *edges_done);

/* mismatches of the reciprocal-plus-fma division against x/d (test helper) */
uint64_t or_check_const_division(uint64_t n, uint64_t seed, const double *divisors, int nd);

#ifdef __cplusplus
}
#endif
#endif
