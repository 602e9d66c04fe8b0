// engine.cuh -- internal interfaces between the engine's translation units.
#pragma once

#include <vector>

#include "common.cuh"
#include "primitives.cuh"

namespace mg {

// Read-only view of a CSR level on the device.  Offsets are 32-bit (every
// level has nnz < 2^32).
struct GraphView {
    uint32_t n = 0;
    uint64_t nnz = 0;
    const uint32_t *off = nullptr;
    const uint32_t *col = nullptr;
    const void *w = nullptr;
    int wk = WK_UNIT;
};

// Degree bins of one level.  Schemes: 0 = 10 local-move bins, 1 = 11
// coarsen-symbolic bins, 2 = 9 coarsen-numeric bins.
struct Bins {
    int scheme = 0;
    int count = 0;
    uint32_t size[11] = {0};
    uint32_t offset[11] = {0};
    uint32_t max_degree = 0;
};

int bin_count(int scheme);
// perm (device, n entries) receives the items bin by bin, ascending id inside
// a bin; sizes/offsets/max degree come back to the host (one sync).
void compute_bins(int scheme, uint32_t n, const uint32_t *d_off, uint32_t *d_perm, Bins &out, cudaStream_t s,
                  PrimWorkspace &ws);

// Accumulators of one sweep (device resident, 64-byte block).
struct SweepAcc {
    unsigned long long sin_u;     // sum of internal weights (integral graphs)
    unsigned long long s2_u;      // sum of sigma^2 (integral graphs)
    unsigned long long distinct;  // candidate (vertex, community) pairs
    unsigned long long moved;     // vertices whose community changed
    double sin_f;                 // same sums for real weights
    double s2_f;
    unsigned long long overflow;  // inserts that found no free slot (must stay 0)
    double pad;
};

// Heavy vertices (last bin) are split into tiers by degree: tier t < 5 is
// served by clusters of 2^t CTAs holding one distributed shared-memory table
// of 2^t * kClusterSlots slots (load <= 1/2); the last tier (giants) by the
// multi-CTA global-table path.
constexpr int kClusterSlots = 16384;
constexpr int kTiers = 6;

// Per-level state of the local-move engine: bins and the heavy-vertex tables.
struct MoveLevel {
    Bins bins;
    uint32_t heavy = 0;            // vertices in the last bin
    uint32_t tier_off[kTiers + 1] = {0};  // heavy vertices by tier (ws.h_tier)
    uint32_t giants = 0;           // vertices on the global-table path
    uint32_t ins_items = 0;        // insert work items (vertex, edge chunk)
    uint32_t eval_items = 0;       // evaluate work items (vertex, slot chunk)
    uint64_t table_slots = 0;
};

struct MoveWorkspace {
    DBuf<uint32_t> perm;
    DBuf<uint32_t> h_tier;         // heavy vertices grouped by tier
    DBuf<uint32_t> h_deg;          // degrees of the heavy vertices
    int max_cluster = 0;           // largest cluster size the device runs (8 or 16)
    // heavy-vertex global tables
    DBuf<uint64_t> h_toff;         // table offset per heavy vertex (H+1)
    DBuf<uint32_t> h_tsize;        // table size per heavy vertex
    DBuf<uint32_t> h_ins;          // insert item offsets (H+1)
    DBuf<uint32_t> h_eval;         // evaluate item offsets (H+1)
    DBuf<uint32_t> h_keys;         // table keys (pool)
    DBuf<double> h_vals;           // table values (pool)
    DBuf<double> h_acc;            // per heavy vertex: e_src, self weight (2H)
    DBuf<unsigned long long> h_best;  // per evaluate item: packed best (gain bits, id) x2
    DBuf<uint64_t> tmp64;
    DBuf<SweepAcc> acc;
    PrimWorkspace prim;
    cudaStream_t streams[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[4] = {nullptr, nullptr, nullptr, nullptr};
    ~MoveWorkspace();
    void init_streams();
};

struct SweepParams {
    int version = 2;
    int up = 1;
    int precision = MG_PREC_FP64;
    double mass = 0;
    int integral = 0;
};

// Constants of the gain of one graph, from its mass (sum of all directed
// weights): m = mass/2 and the correctly rounded reciprocals the exact
// division by m and 2m uses, in FP64 and FP32, and the mass as an integer.
struct GainK {
    double m, two_m, r_m, r_two_m;
    float m_f, two_m_f, r_m_f, r_two_m_f;
    long long mass_i;
};
GainK gain_constants(double mass);

// Batched sweeps run the local move of many graphs packed as one disjoint
// union.  Each graph has a control word:
//   bit 0      active: its vertices take part in the next sweep
//   bits 1-2   assignment buffer the sweep reads (P)
//   bits 3-4   assignment buffer the sweep writes (N)
//   bits 5-6   buffer holding the last accepted assignment (base)
//   bit 7      the next sweep is the first of the phase
//   bit 8      a sigma update is pending
//   bits 9-10  / 11-12  the update moves vertices from buffer / to buffer
constexpr uint32_t kGwActive = 1u, kGwFirst = 1u << 7, kGwUpdate = 1u << 8;
__host__ __device__ inline uint32_t gw_p(uint32_t w) { return (w >> 1) & 3u; }
__host__ __device__ inline uint32_t gw_n(uint32_t w) { return (w >> 3) & 3u; }
__host__ __device__ inline uint32_t gw_base(uint32_t w) { return (w >> 5) & 3u; }
__host__ __device__ inline uint32_t gw_from(uint32_t w) { return (w >> 9) & 3u; }
__host__ __device__ inline uint32_t gw_to(uint32_t w) { return (w >> 11) & 3u; }
__host__ __device__ inline uint32_t gw_make(bool active, uint32_t p, uint32_t n, uint32_t base, bool first,
                                            bool update, uint32_t from, uint32_t to) {
    return (active ? kGwActive : 0u) | (p << 1) | (n << 3) | (base << 5) | (first ? kGwFirst : 0u) |
           (update ? kGwUpdate : 0u) | (from << 9) | (to << 11);
}

struct BatchSweep {
    const uint32_t *perm = nullptr;   // bins 0-8 list (the level's bins give its sizes)
    const uint32_t *pgid = nullptr;   // graph of each entry of perm
    const uint32_t *gid = nullptr;    // graph of each vertex of the union
    const uint32_t *gword = nullptr;  // control word per graph
    const GainK *gk = nullptr;        // gain constants per graph
    uint32_t *C[3] = {nullptr, nullptr, nullptr};
    double *sinv = nullptr;           // out: sum_in contribution per vertex
    const int *up = nullptr;          // sweep direction (device)
};

// Prepare a level: bins (scheme 0) and heavy-vertex tables.
void move_prepare_level(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, cudaStream_t s);
// One local-move sweep P -> N (plus the internal-weight sum of P), device
// accumulators in ws.acc (zeroed by the caller via sweep_reset_acc).
void move_sweep(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                const uint32_t *P, uint32_t *N, const double *k, const double *sigma, cudaStream_t s);
// The same sweep over a batch: per vertex, the graph's control word selects
// the buffers and the gain constants, and sum_in goes to b.sinv.
void move_sweep_batch(const GraphView &g, const MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
                      const BatchSweep &b, const double *k, const double *sigma, cudaStream_t s);
void sweep_reset_acc(MoveWorkspace &ws, cudaStream_t s);
// sum of sigma^2 into ws.acc
void sigma_sumsq(const double *sigma, uint32_t n, int integral, MoveWorkspace &ws, cudaStream_t s);
// sigma += k moved from P[v] to N[v]; counts moved vertices into ws.acc
void sigma_update(const uint32_t *P, const uint32_t *N, const double *k, double *sigma, uint32_t n,
                  MoveWorkspace &ws, cudaStream_t s);
// k_i = row sums; sigma = k; C = identity
void level_init(const GraphView &g, double *k, double *sigma, uint32_t *C, cudaStream_t s);
// Q = sum_in/mass - s2/mass^2 from host-side copy of the accumulators
double modularity_from_acc(const SweepAcc &a, double mass, int integral);

// Coarsening.  out_off/out_col/out_w are resized as needed.
struct CoarsenWorkspace {
    DBuf<uint32_t> flags, newid;
    DBuf<uint64_t> keys, keys_alt;
    DBuf<double> vals, vals_alt;
    DBuf<uint32_t> seg, rowcnt;
    DBuf<uint64_t> u64tmp;
    DBuf<uint32_t> u32tmp;
    PrimWorkspace prim;
};
struct LevelGraph {
    uint32_t n = 0;
    uint64_t nnz = 0;
    DBuf<uint32_t> off, col;
    DBuf<double> w;
    GraphView view() const {
        GraphView v;
        v.n = n;
        v.nnz = nnz;
        v.off = off.get();
        v.col = col.get();
        v.w = w.get();
        v.wk = WK_F64;
        return v;
    }
};
// Dense order-preserving relabel; returns n'.
uint32_t relabel_dense(const uint32_t *C, uint32_t n, uint32_t *C_dense, CoarsenWorkspace &ws, cudaStream_t s);
// Next level from a graph and a dense assignment with n' communities.
void coarsen_level(const GraphView &g, const uint32_t *C_dense, uint32_t n_new, int integral, LevelGraph &out,
                   CoarsenWorkspace &ws, cudaStream_t s, uint64_t *upper_degree_off /* device, may be null */);

// Build a symmetric deduplicated CSR from undirected pairs already on the
// device (self-loops dropped); used by the generators.
void csr_from_device_pairs(uint32_t n, uint64_t m, const uint32_t *u, const uint32_t *v, LevelGraph &out,
                           CoarsenWorkspace &ws, cudaStream_t s);

// device-side helpers
void gather_compose(uint32_t *assign, const uint32_t *map, uint32_t n0, cudaStream_t s);
void fill_identity(uint32_t *C, uint32_t n, cudaStream_t s);

}  // namespace mg
