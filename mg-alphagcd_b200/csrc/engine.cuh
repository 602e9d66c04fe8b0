// engine.cuh -- internal interfaces between the engine's translation units.
#pragma once

#include <cstdlib>
#include <map>
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
    // every row strictly increasing (so no repeated neighbour): generated and
    // coarsened graphs, and uploaded ones that pass the check
    bool sorted_rows = false;
    // integral weights and every entry (u, v, w) matched by an entry (v, u, w)
    // (as multisets): generated graphs, their coarsened levels, and uploaded
    // integral graphs whose fingerprint check passes.  The coarsening then
    // expands every edge from its transposed side (see coarsen_level).
    bool symmetric = false;
};

// Degree bins of one level.  Schemes: 0 = 10 local-move bins, 1 = 11
// coarsen-symbolic bins, 2 = 9 coarsen-numeric bins (the reference's three),
// 3 = the sweep's 19 degree classes (class c holds 2^(c-1) < deg <= 2^c).
constexpr int kMaxBins = 20;
constexpr int kSweepScheme = 3, kSweepClasses = 19;
constexpr int kLightClasses = 13;   // classes 0-12 (deg <= 4096): tile / hash shapes
constexpr int kFirstHeavyClass = 13;
struct Bins {
    int scheme = 0;
    int count = 0;
    uint32_t size[kMaxBins] = {0};
    uint32_t offset[kMaxBins] = {0};
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
// served by clusters of tier_ctas(t) CTAs holding one distributed
// shared-memory table of tier_ctas(t) segments (load <= 1/2); the last tier
// (giants) by the multi-CTA global-table path.
constexpr int kClusterSlots = 16384;
// Slots of one CTA's listed table segment.  (22,528 listed slots of 32-bit
// sums also fit one CTA, which would serve classes 15-17 with 3, 6 and 12
// CTAs instead of 4, 8 and 16; measured on R-MAT-24 the run went 0.52 ->
// 0.69 s.  The dense segments below keep power-of-two clusters and 192 KB.)
template <int WK>
constexpr int kSegSlots = kClusterSlots;
// Dense segments (integral weights): 24,576 slots of a 32-bit key and a
// 32-bit sum (192 KB) per 1,024-thread CTA and no insertion list -- the
// evaluation scans the slots -- at table load <= 2/3, so one CTA holds 16,384
// distinct communities and tiers 1-4 need half the CTAs of listed segments
// (every CTA of a cluster reads the whole row with the own fill).  Tier 0
// (degrees <= 8,192) runs 512-thread CTAs with half a segment.
constexpr int kDenseSlots = 24576;
constexpr int kDenseCapacity = kDenseSlots / 3 * 2;
template <int WK>
constexpr bool kDenseTier(int /*t*/) {
    return kIntg<WK>;
}
// CTAs of the cluster serving heavy tier t (degree class 13 + t, degrees up
// to 2^(13+t)): 1, 2, 4, 8, 16 at table load <= 1/2 with the listed segments,
// 1, 1, 2, 4, 8 with dense segments.
template <int WK>
constexpr int tier_ctas(int t) {
    return kDenseTier<WK>(t)
               ? (int)(((1ull << (13 + t)) + kDenseCapacity - 1) / kDenseCapacity)
               : (int)((2ull * (1ull << (13 + t)) + kSegSlots<WK> - 1) / kSegSlots<WK>);
}
constexpr int kTiers = 6;

// Kernel shapes of the light classes (0-12): T-lane tiles (deg <= T) and
// shared-memory hash tables worked by GT threads per vertex.
enum SweepShape : uint8_t {
    SH_T2, SH_T4, SH_T8, SH_T16, SH_T32,  // tiles
    SH_H32, SH_H64, SH_H128, SH_H256, SH_H512,  // hash, GT threads per vertex
    SH_W,  // a warp per batch of vertices, a table per vertex (classes 5-10)
    SH_COUNT
};
// largest degree a shape serves
inline uint32_t shape_capacity(int sh) {
    switch (sh) {
        case SH_T2: return 2;
        case SH_T4: return 4;
        case SH_T8: return 8;
        case SH_T16: return 16;
        case SH_T32: return 32;
        case SH_H32: return 512;
        case SH_H64: return 1024;
        case SH_W: return 1024;
        default: return 4096;
    }
}
const char *shape_name(int sh);
// the shapes used when nothing has been tuned
int default_shape(int cls);

// Per-level state of the local-move engine: degree classes, the shape of
// every light class, and the heavy-vertex tables.
struct MoveLevel {
    Bins bins;                     // sweep classes (scheme 3)
    uint8_t shape[kLightClasses] = {0};
    uint32_t heavy = 0;            // vertices of the heavy classes (13-18)
    const uint32_t *heavy_list = nullptr;  // those vertices, by class (a range of the level's perm)
    uint32_t tier_off[kTiers + 1] = {0};  // heavy vertices by tier (in heavy_list)
    uint32_t giants = 0;           // vertices on the global-table path
    uint32_t ins_items = 0;        // insert work items (vertex, edge chunk)
    uint32_t eval_items = 0;       // evaluate work items (vertex, slot chunk)
    uint64_t table_slots = 0;
};

// Autotuner table: the fastest shape of a light class, keyed by the kernel
// weight kind, precision, version, single / batched sweep, class and the
// class size (log2 bucket).  Filled by timing the candidate shapes of a class
// on the level's first sweep; the sweep's results do not depend on the shapes.
struct TuneEntry {
    uint8_t shape;
    float us;  // timed duration of the chosen shape
};
struct TuneTable {
    int mode = MG_TUNE_ON;
    // print every timed candidate to stderr (environment variable MG_TUNE_LOG=1)
    bool log = getenv("MG_TUNE_LOG") != nullptr && getenv("MG_TUNE_LOG")[0] == '1';
    std::map<uint32_t, TuneEntry> entries;
    unsigned long long tuned = 0;  // classes tuned (timed) so far
    static uint32_t key(int wk, int prec, int ver, int bt, int cls, uint32_t size) {
        const uint32_t bucket = size ? 31u - (uint32_t)__builtin_clz(size) : 0u;
        return (uint32_t)wk | (uint32_t)prec << 3 | (uint32_t)ver << 5 | (uint32_t)bt << 7 | (uint32_t)cls << 8 |
               bucket << 13;
    }
};
constexpr uint32_t kTuneMinVertices = 4096;  // smaller classes keep the default shape

struct MoveWorkspace {
    DBuf<uint32_t> perm;
    DBuf<uint2> rows;              // {off[perm[q]], off[perm[q] + 1]} per class-list entry q
    int max_cluster = 0;           // largest cluster size the device runs (8 or 16)
    // heavy-vertex policy (mg_sweep_options): first degree class worked by the
    // global-table path (13..18), and the cluster-table fill (MG_FILL_*)
    int giant_class = kFirstHeavyClass + kTiers - 1;
    int cluster_fill = MG_FILL_AUTO;
    int coarsen_combine = MG_COMBINE_AUTO;  // MG_COMBINE_*, read by the coarsening of a run
    int first_sweep_kernels = 1;            // table-free kernels for a level's first sweep
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
    DBuf<SweepAcc> tune_acc;       // sums of the autotuner's timing runs (discarded)
    TuneTable tune;
    PrimWorkspace prim;
    // stream 0: heavy tiers; streams 1..light_streams: the light classes and
    // the class-13 tier, so that one class's tail overlaps the others (one by
    // default: with the dense cluster tiers, R-MAT-24 ran 0.4593 s on one,
    // 0.4635 s on two, 0.4605 s on three, 0.4635 s on four)
    static constexpr int kStreams = 8;
    static constexpr int kDefaultLightStreams = 1;
    cudaStream_t streams[kStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kStreams] = {};
    int light_streams = kDefaultLightStreams;
    cudaEvent_t ev_tune[2] = {nullptr, nullptr};  // timing events of the autotuner
    ~MoveWorkspace();
    void init_streams();
};

struct SweepParams {
    int version = 2;
    int up = 1;
    int precision = MG_PREC_FP64;
    double mass = 0;
    int integral = 0;
    // communities repeat among neighbours: the table kernels add a thread's
    // consecutive edges into one community in a register before inserting
    // (fewer shared-memory adds to one slot); set from the previous sweep's
    // distinct candidates per edge (never on the first sweep of a phase,
    // where every community is one vertex)
    int agg = 0;
    // cluster tables: split fill with warp combining (MG_FILL_SPLIT) instead
    // of the own fill
    int split = 0;
    // the level's first sweep from the identity assignment with sigma = k
    // (single-graph runs): every neighbour is its own candidate community
    int first = 0;
};
// split fill only when forced: the own fill measured faster on R-MAT-24 at
// every level (also against splitting the sweeps where communities repeat)
inline int sweep_split(const MoveWorkspace &ws, int /*agg*/) { return ws.cluster_fill == MG_FILL_SPLIT; }
// combining in the coarsening of a run: automatic when the phase's last sweep
// saw at most one distinct candidate community per 4 edges
inline bool coarsen_combine(const MoveWorkspace &ws, unsigned long long distinct, uint64_t nnz) {
    return ws.coarsen_combine == MG_COMBINE_ON ||
           (ws.coarsen_combine == MG_COMBINE_AUTO && 4 * distinct <= nnz);
}

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
// Shapes of the level's light classes from the tuning table; with MG_TUNE_ON,
// classes missing from it are timed now with the sweep's arguments (P, N, k,
// sigma as the next sweep will use them: the timing runs write the same N).
// With timing = false the table is only read (classes missing from it keep
// the built-in shapes).
void move_tune(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p, const uint32_t *P,
               uint32_t *N, const double *k, const double *sigma, cudaStream_t s, bool timing = true);
void move_tune_batch(const GraphView &g, MoveLevel &lvl, MoveWorkspace &ws, const SweepParams &p,
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
    DBuf<uint32_t> tcount;  // combined entries per expansion tile
    // member order of a symmetric coarsening: per member (vertices sorted by
    // community) its row start, its community, and its row's offset in the
    // member-ordered expansion
    DBuf<uint32_t> msrc, mcom, voff;
    PrimWorkspace prim;
};
// A device CSR level: f64 weights (w, wk = WK_F64), or exact 32-bit integer
// weights (wi, wk = WK_U32) for the coarsened levels of integral graphs.
struct LevelGraph {
    uint32_t n = 0;
    uint64_t nnz = 0;
    DBuf<uint32_t> off, col;
    DBuf<double> w;
    DBuf<uint32_t> wi;
    int wk = WK_F64;
    bool symmetric = false;  // coarsened from a symmetric integral graph
    GraphView view() const {
        GraphView v;
        v.n = n;
        v.nnz = nnz;
        v.off = off.get();
        v.col = col.get();
        v.w = wk == WK_U32 ? (const void *)wi.get() : (const void *)w.get();
        v.wk = wk;
        v.sorted_rows = true;  // generated and coarsened levels have sorted, deduplicated rows
        v.symmetric = symmetric;
        return v;
    }
};
// The weights of a level as doubles (device, nnz entries).
void level_weights_f64(const GraphView &g, double *out, cudaStream_t s);
// Dense order-preserving relabel; returns n'.
uint32_t relabel_dense(const uint32_t *C, uint32_t n, uint32_t *C_dense, CoarsenWorkspace &ws, cudaStream_t s);
// Next level from a graph and a dense assignment with n' communities.
// combine: merge equal keys within each warp's 32 edges before sorting (pays
// when communities repeat inside rows); the result does not depend on it.
void coarsen_level(const GraphView &g, const uint32_t *C_dense, uint32_t n_new, int integral, LevelGraph &out,
                   CoarsenWorkspace &ws, cudaStream_t s, uint64_t *upper_degree_off /* device, may be null */,
                   bool combine = false);

// Build a symmetric deduplicated CSR from undirected pairs already on the
// device (self-loops dropped); used by the generators.  With pair weights w
// (equal for duplicate pairs), out.w receives the weight of every entry.
void csr_from_device_pairs(uint32_t n, uint64_t m, const uint32_t *u, const uint32_t *v, LevelGraph &out,
                           CoarsenWorkspace &ws, cudaStream_t s, const double *w = nullptr);

// device-side helpers
void gather_compose(uint32_t *assign, const uint32_t *map, uint32_t n0, cudaStream_t s);
void fill_identity(uint32_t *C, uint32_t n, cudaStream_t s);

}  // namespace mg
