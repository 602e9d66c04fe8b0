/*
 * mgagcd.h -- C ABI of the B200 Louvain engine (libmgagcd.so).
 *
 * The reference (MG-alphaGCD) has no plugin or FFI layer: its boundary is the
 * in-process C++ call chain driven by the MG_GCD binary (src/main.cu:118-131).
 * Each entry point below names the reference interface it replaces.  All
 * entry points return mg_status (never exit, never throw across the ABI);
 * mg_last_error() gives the text of the last failure on a context.
 *
 * Ownership: the library owns every mg_graph / mg_result it returns; the
 * caller releases them with the matching *_destroy.  Host buffers passed in
 * are only read during the call; output buffers are sized by the caller as
 * documented.  A context is bound to one CUDA device and one host thread at a
 * time.
 */
#ifndef MGAGCD_H
#define MGAGCD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MG_OK = 0,
    MG_ERR_INVALID = 1,     /* bad argument / handle */
    MG_ERR_CUDA = 2,        /* CUDA runtime error */
    MG_ERR_OOM = 3,         /* device or host allocation failed / over budget */
    MG_ERR_IO = 4,          /* file cannot be opened */
    MG_ERR_FORMAT = 5,      /* malformed .mtx input */
    MG_ERR_UNSUPPORTED = 6, /* size or mode outside what the engine supports */
    MG_ERR_TIMEOUT = 7,     /* a bounded device wait or probe gave up */
    MG_ERR_CANCELLED = 8    /* job cancelled */
} mg_status;

typedef struct mg_ctx mg_ctx;
typedef struct mg_graph mg_graph;
typedef struct mg_result mg_result;

/* weight element types for mg_graph_from_csr */
enum { MG_WEIGHT_UNIT = 0, MG_WEIGHT_F32 = 1, MG_WEIGHT_F64 = 2 };

/* precision modes of the local-move gain (mg_run_opts.precision) */
enum {
    MG_PREC_FP64 = 0,  /* the reference's double arithmetic (default) */
    MG_PREC_INT64 = 1, /* exact integer gain comparison; integral weights only */
    MG_PREC_FP32 = 2   /* single-precision gains, double sigma_tot and modularity */
};

typedef struct {
    int device;              /* CUDA device ordinal (default 0) */
    int verbose;             /* print the reference's tables to stdout */
    size_t hbm_budget_bytes; /* 0 = no limit */
} mg_opts;

const char *mg_status_string(mg_status s);
const char *mg_version(void);

/* Context.  Replaces the process setup of src/main.cu:28-59 (device select);
 * no MPI / NVSHMEM init is needed on one GPU. */
mg_status mg_init(mg_ctx **ctx, const mg_opts *opts /* may be NULL */);
mg_status mg_destroy(mg_ctx *ctx);
const char *mg_last_error(const mg_ctx *ctx);

/* ---- graphs -------------------------------------------------------------- */

/* Copy a symmetric CSR from host memory into library-owned device memory.
 * offsets[n+1] (uint64), cols[nnz] (uint32), weights per weight_type (NULL
 * with MG_WEIGHT_UNIT).  nnz = offsets[n] must be < 2^32.
 * Replaces HostGraph + GpuGraph + edge_partition::partitioner for one GPU
 * (src/graph/host_graph.cpp:3, src/graph/gpu_graph.cu:3,
 *  src/partition/edge_partition.cu:26). */
mg_status mg_graph_from_csr(mg_ctx *ctx, uint32_t n, const uint64_t *offsets, const uint32_t *cols,
                            const void *weights, int weight_type, mg_graph **out);

/* Same, with the arrays already in device memory (copied device-to-device). */
mg_status mg_graph_from_device_csr(mg_ctx *ctx, uint32_t n, uint64_t nnz, const uint32_t *d_offsets32,
                                   const uint32_t *d_cols, const void *d_weights, int weight_type,
                                   mg_graph **out);

/* Load a Matrix Market file with the reference's rules.
 * Replaces loadMMSparseMatrix / init_data_from_mtx (src/mmio/mmio_wrapper.cu:76-301). */
mg_status mg_graph_from_mtx(mg_ctx *ctx, const char *path, mg_graph **out);

/* ---- host-side loading (no GPU needed) ------------------------------------ */

/* A symmetric CSR in host memory produced by the .mtx loader. */
typedef struct mg_host_csr mg_host_csr;

enum {
    MG_LOAD_CACHE_READ = 1,  /* use "<path>.mgcsr" when it matches the file's size and mtime */
    MG_LOAD_CACHE_WRITE = 2  /* write "<path>.mgcsr" after parsing (a failed write is not an error) */
};

/* Parse a Matrix Market file with the same rules as mg_graph_from_mtx
 * (src/mmio/mmio_wrapper.cu:76-295): memory-mapped, parsed by all host
 * threads, rows in file order.  Symmetric files give unit weights (the
 * reference forces 1.0, :141-142) and no weight array. */
mg_status mg_csr_from_mtx(const char *path, int flags, mg_host_csr **out);
/* Sizes; weighted = 0 when every weight is 1; from_cache = 1 when the arrays
 * were mapped from the binary cache; cache_written = 1 when this load wrote it.
 * Any pointer may be NULL. */
mg_status mg_csr_info(const mg_host_csr *c, uint32_t *n, uint64_t *nnz, int *weighted, int *from_cache,
                      int *cache_written);
/* Borrowed views, valid until mg_csr_free: offsets[n+1], cols[nnz], weights[nnz] (NULL when unweighted). */
mg_status mg_csr_arrays(const mg_host_csr *c, const uint64_t **offsets, const uint32_t **cols,
                        const double **weights);
void mg_csr_free(mg_host_csr *c);

/* mg_graph_from_mtx with cache flags (MG_LOAD_*). */
mg_status mg_graph_from_mtx_ex(mg_ctx *ctx, const char *path, int flags, mg_graph **out);

/* Seeded synthetic graphs generated on the device (integer-only RNG; the
 * same seed gives the same graph as the CPU generators of the test oracle).
 * Replaces HostGraph::randomly_generate_graph (src/graph/host_graph.cpp:38-77). */
mg_status mg_graph_generate_rmat(mg_ctx *ctx, int scale, int edge_factor, double a, double b, double c,
                                 uint64_t seed, mg_graph **out);
mg_status mg_graph_generate_sbm(mg_ctx *ctx, uint32_t n, uint32_t blocks, double mean_degree,
                                double intra_frac, uint64_t seed, mg_graph **out);
/* Chung-Lu power-law graph: expected degree of vertex i proportional to
 * (i + i0)^(-1/(exponent-1)), mean mean_degree, capped at max_degree;
 * lognormal = 1 gives every edge a weight lognormal(0, 1) rounded to float
 * (stored as f32), else unit weights.  The same seed gives the same topology
 * with and without weights, and the same topology as the test oracle's
 * generator. */
mg_status mg_graph_generate_chunglu(mg_ctx *ctx, uint32_t n, double exponent, double mean_degree,
                                    double max_degree, int lognormal, uint64_t seed, mg_graph **out);

/* n, nnz, mass (sum of all directed weights, src/graph/host_graph.cpp:112-115),
 * integral (1 when every weight is a non-negative integer and mass < 2^32). */
mg_status mg_graph_info(const mg_graph *g, uint32_t *n, uint64_t *nnz, double *mass, int *integral);
/* Row properties the engine found (no reference counterpart): sorted_rows = 1
 * when every row is strictly increasing (generated and coarsened graphs, and
 * uploads that pass the check: the first sweep of a level then runs
 * table-free); symmetric = 1 when the weights are integral and the entries
 * are, as a multiset, their own transposes (generated graphs, their
 * coarsened levels, and uploads whose two 64-bit fingerprints agree: the
 * coarsening then sorts only the high half of its keys).  Either pointer may
 * be NULL. */
mg_status mg_graph_properties(const mg_graph *g, int *sorted_rows, int *symmetric);
/* Copy the CSR back to host buffers (offsets[n+1], cols[nnz], weights[nnz]
 * as double; any pointer may be NULL). */
mg_status mg_graph_copy_csr(const mg_graph *g, uint64_t *offsets, uint32_t *cols, double *weights);
mg_status mg_graph_destroy(mg_graph *g);

/* ---- stage hooks (the reference's stage boundaries) ----------------------- */

/* Degree binning of the graph's rows.  scheme 0: 10 local-move bins
 * (src/bin/BIN.cu:468-499), 1: 11 coarsen-symbolic bins (:501-540),
 * 2: 9 coarsen-numeric bins (:542-575).  sizes/offsets: 11 slots (unused
 * slots zero); perm[n]: items bin by bin, ascending id inside a bin. */
mg_status mg_bins(mg_graph *g, int scheme, uint32_t *sizes, uint32_t *offsets, uint32_t *perm,
                  uint32_t *max_degree);
/* Same over an arbitrary offsets array (degree of item i = offsets[i+1]-offsets[i]),
 * as BIN::bin_create(com_degree, ...) is used on community degrees. */
mg_status mg_bins_offsets(mg_ctx *ctx, int scheme, uint32_t n, const uint64_t *offsets, uint32_t *sizes,
                          uint32_t *bin_offsets, uint32_t *perm, uint32_t *max_degree);

/* One local-move sweep from assignment C with community weights sigma and
 * vertex weights k (host buffers of n), writing C_new.  version 2 (default
 * reference behaviour) or 1; up = 1 for an "up" iteration.
 * Replaces louvain::calculate_eicj_and_move_vertex_bin (src/louvain/louvain.cu:1032-1296,
 * src/louvain/louvain_gl.cu:1018).  distinct (optional) receives the number of
 * distinct (vertex, neighbour community) candidate pairs. */
mg_status mg_local_move(mg_graph *g, int version, int up, int precision, const uint32_t *C,
                        const double *sigma, const double *k, uint32_t *C_new, uint64_t *distinct);

/* One local-move sweep that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc, such as a
 * serving process that has handed its whole HBM budget to its own pool, or
 * code that must not enter the CUDA allocator.  Everything is in device
 * memory owned by the caller: the CSR (d_offsets[n+1] as uint32, d_cols,
 * d_weights or NULL for unit weights), the assignment d_C, sigma d_sigma, vertex
 * weights d_k (n each) and the output d_C_new (n).  mass = sum of all
 * weights.  Results equal mg_local_move (FP64 gains) for integral weights.
 * Work is queued on `stream` (a cudaStream_t, NULL = default stream); the call
 * waits for the stream once, to read the graph's maximum degree, so it must
 * not be called while that stream is being captured into a CUDA graph.
 * Scratch: the per-block hash tables live in one static 16 MiB device array
 * that every GPU loading the library holds until exit; each vertex uses a
 * table sized by its own degree.  A graph whose maximum degree needs a table
 * beyond it (a degree above 524,287) is rejected with MG_ERR_UNSUPPORTED.
 * The first call on a device looks up that array's device address (a
 * one-time set-up per device).  All calls share the array and clear it on
 * entry, so calls that overlap on the GPU race with each other.  Errors are
 * reported by mg_last_error(NULL). */
mg_status mg_local_move_noalloc(uint32_t n, const uint32_t *d_offsets, const uint32_t *d_cols,
                                const double *d_weights, double mass, const uint32_t *d_C,
                                const double *d_sigma, const double *d_k, uint32_t *d_C_new,
                                int version, int up, void *stream);

/* Modularity of an assignment (src/louvain/louvain.cu:105-238), sigma_tot
 * computed from C. */
mg_status mg_modularity(mg_graph *g, const uint32_t *C, double *q);

/* Coarsen by assignment C: dense order-preserving relabel (written to
 * C_dense[n] if not NULL) and the next-level graph with rows sorted by
 * neighbour community, self-loops kept.
 * Replaces coarsen_graph_mg::coarsen_graph (src/coarsen_graph/coarsen_graph_mg.cu:2054-2240). */
mg_status mg_coarsen(mg_graph *g, const uint32_t *C, uint32_t *C_dense, mg_graph **out);

/* ---- full Louvain ----------------------------------------------------------- */

typedef struct {
    int version;       /* 0, 1 or 2 (src/main.cu:118-131); 0 behaves as 2 on one GPU */
    double threshold;  /* default 1e-6 (src/main.cu:21) */
    int max_phases;    /* default 1000 (src/main.cu:23) */
    int precision;     /* MG_PREC_* */
    int verbose;       /* print the reference's per-phase tables */
    int keep_levels;   /* 1: keep the dendrogram, every level's community map (mg_result_level_map);
                          2: also every level's graph on the host (mg_result_level_csr) */
} mg_run_opts;

typedef struct {
    double modularity;       /* final Q */
    int phases;              /* coarsening steps taken */
    int levels;              /* phases started */
    int iterations;          /* local-move iterations as the reference counts them */
    uint32_t communities;    /* final community count */
    double seconds_total;    /* device time of the whole run */
    double seconds_local_move;
    double seconds_coarsen;
    uint64_t edges_swept;    /* sum over sweeps of the level's nnz */
    uint64_t phase0_edges_swept;
    double phase0_seconds;
    uint64_t distinct_pairs; /* sum over sweeps of the candidate pairs */
    double seconds_sweep_kernels; /* device time of the local-move kernels alone */
    double sweep_bytes;      /* algorithmic bytes of those sweeps: 12E + 24V + 8D each */
    uint64_t kernel_launches; /* engine kernels launched during the run */
    uint64_t sweeps;         /* edge passes run (iterations + one per phase) */
} mg_summary;

/* Run Louvain to convergence.  Replaces louvain::run / louvain_gl::run /
 * louvain_baseline::run (src/louvain/louvain.cu:1401-1715). */
mg_status mg_louvain_run(mg_graph *g, const mg_run_opts *opts /* may be NULL */, mg_result **out);
mg_status mg_result_summary(const mg_result *r, mg_summary *s);
/* composed final community of every input vertex (dense ids), n entries */
mg_status mg_result_assignment(const mg_result *r, uint32_t *out);
/* vertex count at the start of each phase; *count receives the number */
mg_status mg_result_level_sizes(const mg_result *r, uint32_t *out, int max, int *count);
/* Dendrogram of a run with keep_levels = 1: the community map of level
 * `level` (0 = the input graph), one id in [0, size of the next level) per
 * vertex of that level.  Composing the maps of levels 0 .. count-1 gives
 * mg_result_assignment; the reference keeps only its last level
 * (src/louvain/louvain.cu:1674-1693).  *size = vertices of the level; `out`
 * (may be NULL) receives min(size, max) entries.  MG_ERR_INVALID when the
 * run did not keep levels or `level` is out of range. */
mg_status mg_result_level_map(const mg_result *r, int level, uint32_t *out, uint32_t max, uint32_t *size);
/* The graph level `level` worked on, for a run with keep_levels = 2 (level 0
 * = the input graph, level l = the coarsened graph of phase l - 1, rows
 * sorted by neighbour community): n, nnz and, for non-NULL pointers,
 * offsets[n+1], cols[nnz], weights[nnz] (double; 1 for unit weights).  The
 * reference coarsens its GpuGraph in place and keeps no level
 * (src/coarsen_graph/coarsen_graph_mg.cu:2224-2228).  MG_ERR_INVALID when
 * the run did not keep level graphs or `level` is out of range. */
mg_status mg_result_level_csr(const mg_result *r, int level, uint32_t *n, uint64_t *nnz, uint64_t *offsets,
                              uint32_t *cols, double *weights);
/* the reference's printed table as rows {phase, loop, Q, dQ} */
mg_status mg_result_trace(const mg_result *r, double *rows4, int max_rows, int *count);
mg_status mg_result_destroy(mg_result *r);

/* ---- autotuner -------------------------------------------------------------------
 * No reference counterpart (the reference's bin thresholds and kernel shapes
 * are fixed, src/bin/BIN.cu:72-92).  The local move groups vertices in degree
 * classes (class c: 2^(c-1) < degree <= 2^c) and works each class up to 4096
 * with a kernel shape: T-lane tiles or shared-memory tables with 32 to 512
 * threads per vertex.  Any shape whose table holds the class gives the same
 * result, so the shape per class is picked by timing: the first sweep of a
 * level times the candidate shapes of each class of at least 4096 vertices that
 * is not yet in the context's table, and the fastest is stored (keyed by weight
 * kind, precision, version, single / batched sweep, class and class size) and
 * reused.  MG_TUNE_OFF uses the built-in shapes, MG_TUNE_CACHED the table
 * without timing anything new, MG_TUNE_ON (default) also fills it. */
enum { MG_TUNE_OFF = 0, MG_TUNE_CACHED = 1, MG_TUNE_ON = 2 };
mg_status mg_tune_mode(mg_ctx *ctx, int mode);
/* The table as text, one entry per line:
 * "<weight kind> <precision> <version> <batched> <class> <size bucket> <shape> <microseconds>".
 * *len receives the length; buf (capacity cap) may be NULL. */
mg_status mg_tune_table(mg_ctx *ctx, char *buf, size_t cap, size_t *len);
/* Save / load the table (same text). Loading merges into the context's table. */
mg_status mg_tune_save(mg_ctx *ctx, const char *path);
mg_status mg_tune_load(mg_ctx *ctx, const char *path);

/* ---- heavy-vertex policy ----------------------------------------------------------
 * Where the reference sends every vertex above degree 4094 to one global-table
 * kernel (calculate_eicj_and_move_vertex_gl_bk, src/louvain/louvain.cu:810-1030,
 * dispatched at :1257-1285), the engine splits them by degree class: classes
 * 13..17 (degree 4,097..131,072) go to thread-block-cluster tables of 1..16 CTAs,
 * class 18 (above 131,072) to global-memory tables.  Every choice below gives
 * the same result (bit for bit on integral weights); they exist for tuning and
 * so that tests can force each path. */
enum {
    MG_FILL_AUTO = 0,  /* the engine's choice: the own fill (measured faster on R-MAT-24 at every level) */
    MG_FILL_OWN = 1,   /* every CTA of a cluster reads the whole row and inserts the communities it owns */
    MG_FILL_SPLIT = 2  /* the CTAs split the row; equal communities combined in the warp; inserts via DSMEM */
};
/* Coarsening (coarsen_graph_mg::coarsen_graph, src/coarsen_graph/coarsen_graph_mg.cu:2054-2240)
 * turns every edge into a (community, neighbour community) key and sorts the
 * keys; with combining, the 32 edges a warp holds are first merged by key, so
 * the sort sees far fewer keys where communities repeat inside rows.  The
 * next-level graph is the same either way. */
enum {
    MG_COMBINE_AUTO = 0, /* in a run: combine when the phase's last sweep saw few distinct candidates; mg_coarsen: off */
    MG_COMBINE_OFF = 1,
    MG_COMBINE_ON = 2
};
typedef struct {
    int cluster_fill;    /* MG_FILL_* */
    int giant_class;     /* degree classes >= this (13..18) take the global-table path; 0 = default (18) */
    int coarsen_combine; /* MG_COMBINE_* */
    int light_streams;   /* streams the light degree classes are spread over, 1..7 (0 = default 1) */
    int table_first_sweep; /* 1: a level's first sweep uses the table kernels too (default 0: every
                              community is one vertex there, so it runs table-free kernels) */
} mg_sweep_opts;
/* Set the context's policy (opts NULL = defaults); applies to later sweeps and runs. */
mg_status mg_sweep_options(mg_ctx *ctx, const mg_sweep_opts *opts);

/* ---- fault injection (test hook) ----------------------------------------------
 * No reference counterpart (the reference exits on any CUDA error,
 * include/common.h:53-83).  Arms a process-wide countdown: the nth device
 * allocation the library makes from now on fails as if cudaMalloc had run out
 * of memory (once; nth = 0 disarms).  *pending (may be NULL) receives what was
 * left of the previous countdown (0 = it fired or was never armed).  The
 * entry point that hits it returns MG_ERR_OOM with text, releases what it
 * allocated, and the context stays usable.  No GPU fault is involved. */
mg_status mg_test_fail_allocation(uint64_t nth, uint64_t *pending);

/* ---- batched form --------------------------------------------------------------
 * No reference counterpart: the reference runs one graph per process.  A batch
 * packs many independent graphs as one disjoint union on the device and runs
 * louvain::run's control flow (src/louvain/louvain.cu:1401-1715) for every
 * graph at once: one set of kernel launches per sweep covers all graphs, each
 * graph keeps its own mass, gain constants, modularity, accept / reject
 * decisions and phase exit, so each result is the one mg_louvain_run gives
 * for that graph alone (bit for bit on integral weights). */
typedef struct mg_batch mg_batch;
typedef struct mg_batch_result mg_batch_result;

/* parameters of one seeded SBM graph (mg_graph_generate_sbm) */
typedef struct {
    uint32_t n;
    uint32_t blocks;
    double mean_degree;
    double intra_frac;
    uint64_t seed;
} mg_sbm_params;

/* Draw per-graph SBM parameters on the host: n log-uniform in [n_min, n_max],
 * blocks uniform in [blocks_min, min(blocks_max, n)], mean degree uniform in
 * [deg_min, deg_max], intra-community fraction uniform in [intra_min,
 * intra_max], graph seeds derived from seed.  Deterministic in seed. */
mg_status mg_batch_draw_sbm_params(uint32_t graphs, uint32_t n_min, uint32_t n_max, uint32_t blocks_min,
                                   uint32_t blocks_max, double deg_min, double deg_max, double intra_min,
                                   double intra_max, uint64_t seed, mg_sbm_params *out);
/* Generate graph g of the batch exactly as mg_graph_generate_sbm(params[g]). */
mg_status mg_batch_generate_sbm(mg_ctx *ctx, uint32_t graphs, const mg_sbm_params *params, mg_batch **out);

/* one seeded generated graph: an SBM (mg_graph_generate_sbm) or an R-MAT
 * graph (mg_graph_generate_rmat) */
enum { MG_GEN_SBM = 0, MG_GEN_RMAT = 1 };
typedef struct {
    int kind;            /* MG_GEN_* */
    uint32_t n;          /* SBM: vertices */
    uint32_t blocks;     /* SBM: planted communities */
    double mean_degree;  /* SBM */
    double intra_frac;   /* SBM */
    int scale;           /* R-MAT: 2^scale vertices */
    int edge_factor;     /* R-MAT: pairs per vertex */
    double a, b, c;      /* R-MAT quadrant probabilities */
    uint64_t seed;
} mg_gen_params;
/* Generate graph g of the batch exactly as the single-graph generator of its kind. */
mg_status mg_batch_generate(mg_ctx *ctx, uint32_t graphs, const mg_gen_params *params, mg_batch **out);
/* Pack host graphs: graph g owns vertices [vertex_offsets[g], vertex_offsets[g+1])
 * of the packed rows; row v's entries are [offsets[v], offsets[v+1]) (64-bit,
 * packed over all graphs); cols hold graph-local vertex ids.  weights as in
 * mg_graph_from_csr (NULL = unit). */
mg_status mg_batch_from_csr(mg_ctx *ctx, uint32_t graphs, const uint64_t *vertex_offsets, const uint64_t *offsets,
                            const uint32_t *cols, const void *weights, int weight_type, mg_batch **out);
/* total vertices / entries of the batch */
mg_status mg_batch_info(const mg_batch *b, uint32_t *graphs, uint64_t *n, uint64_t *nnz);
/* one graph: vertices, entries, mass */
mg_status mg_batch_graph_info(const mg_batch *b, uint32_t g, uint32_t *n, uint64_t *nnz, double *mass);
mg_status mg_batch_destroy(mg_batch *b);

enum {
    MG_BATCH_GRAPHS = 1 /* run each phase's iterations as one CUDA graph with a device-side loop */
};

typedef struct {
    double modularity;
    uint32_t n;
    uint64_t nnz;
    int phases;
    int levels;
    uint64_t iterations;
    uint32_t communities;
} mg_batch_graph_summary;

/* Run Louvain on every graph of the batch.  flags: MG_BATCH_*. */
mg_status mg_batch_run(mg_batch *b, const mg_run_opts *opts /* may be NULL */, int flags, mg_batch_result **out);
/* totals of the run (seconds, sweeps, edges, launches); per-graph fields
 * (modularity, phases, levels, iterations, communities) are left zero */
mg_status mg_batch_result_summary(const mg_batch_result *r, mg_summary *s);
mg_status mg_batch_result_graph(const mg_batch_result *r, uint32_t g, mg_batch_graph_summary *out);
/* final community (dense, graph-local) of every vertex of graph g: n_g entries */
mg_status mg_batch_result_assignment(const mg_batch_result *r, uint32_t g, uint32_t *out);
mg_status mg_batch_result_destroy(mg_batch_result *r);

/* ---- serving ---------------------------------------------------------------------
 * No reference counterpart.  A server admits Louvain jobs from any number of
 * host threads and runs them with continuous batching: `slots` worker
 * threads, each with its own context (streams and workspaces) and an equal
 * share of the HBM budget, take the queued jobs in arrival order as soon as
 * they are free, pack as many as fit their share into one batch
 * (mg_batch_run) and run it; batches of different slots overlap on the GPU.
 * A job is done as soon as its own graph finishes inside its batch.  Each
 * job's result equals mg_louvain_run on its graph alone (bit for bit on
 * integral weights).  All mg_serve_* calls are thread-safe. */
typedef struct mg_server mg_server;

typedef struct {
    int device;
    int slots;                 /* batches in flight (default 4) */
    size_t hbm_budget_bytes;   /* shared equally by the slots (default 150e9) */
    uint32_t max_batch_jobs;   /* jobs per batch at most (default 4096) */
    int batch_flags;           /* MG_BATCH_* (default MG_BATCH_GRAPHS) */
} mg_serve_opts;

enum { MG_JOB_QUEUED = 0, MG_JOB_RUNNING = 1, MG_JOB_DONE = 2, MG_JOB_FAILED = 3, MG_JOB_CANCELLED = 4 };

typedef struct {
    int state;                     /* MG_JOB_* */
    mg_status status;              /* of a failed job */
    mg_batch_graph_summary graph;  /* result of a done job */
    double submitted_s;            /* times in seconds since the server started */
    double started_s;
    double finished_s;
    uint64_t batch;                /* batch the job ran in (1, 2, ...) */
    uint32_t batch_jobs;           /* jobs in that batch */
} mg_job_info;

typedef struct {
    uint64_t submitted, completed, failed, cancelled, queued, running;
    uint64_t batches;
    double elapsed_s;              /* since the server started */
    double jobs_per_s;             /* completed / elapsed */
    double p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s; /* submit -> done */
    size_t budget_bytes;
    size_t reserved_bytes;         /* estimates of the jobs running now */
} mg_serve_counters;

/* Start the worker slots (opts may be NULL for the defaults). */
mg_status mg_serve_start(const mg_serve_opts *opts, mg_server **out);
/* Queue a generated graph; opts NULL = defaults; keep_assignment: keep the
 * final assignment for mg_serve_assignment.  Jobs larger than one slot's
 * budget are refused with MG_ERR_OOM. */
mg_status mg_serve_submit(mg_server *s, const mg_gen_params *job, const mg_run_opts *opts, int keep_assignment,
                          uint64_t *id);
/* Queue a host CSR graph (copied at submit; arguments as mg_graph_from_csr). */
mg_status mg_serve_submit_csr(mg_server *s, uint32_t n, const uint64_t *offsets, const uint32_t *cols,
                              const void *weights, int weight_type, const mg_run_opts *opts, int keep_assignment,
                              uint64_t *id);
mg_status mg_serve_poll(mg_server *s, uint64_t id, mg_job_info *info);
/* Wait until the job is done, failed or cancelled; MG_ERR_TIMEOUT after timeout_s. */
mg_status mg_serve_wait(mg_server *s, uint64_t id, double timeout_s, mg_job_info *info);
/* The kept assignment of a done job (graph.n entries). */
mg_status mg_serve_assignment(mg_server *s, uint64_t id, uint32_t *out);
/* Cancel a queued job (running jobs finish). */
mg_status mg_serve_cancel(mg_server *s, uint64_t id);
/* Forget a finished job. */
mg_status mg_serve_release(mg_server *s, uint64_t id);
mg_status mg_serve_stats(mg_server *s, mg_serve_counters *out);
const char *mg_serve_last_error(mg_server *s);
/* Cancel the queued jobs, wait for the running batches, stop the workers. */
mg_status mg_serve_stop(mg_server *s);

#ifdef __cplusplus
}
#endif
#endif
