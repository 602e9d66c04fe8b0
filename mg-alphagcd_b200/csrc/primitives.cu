// primitives.cu -- device-wide exclusive scan (reduce-then-scan over tiles)
// and stable LSD radix sort (8-bit digits, warp match_any ranking).
#include "primitives.cuh"

namespace mg {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ __forceinline__ T block_exclusive_sum(T v, T *smem_warp, T *total) {
    // smem_warp: 8 entries
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) smem_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T x = lane < (kScanThreads / 32) ? smem_warp[lane] : T(0);
        T xi = x;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane < (kScanThreads / 32)) smem_warp[lane] = xi - x;
        if (lane == (kScanThreads / 32) - 1) *total = xi;
    }
    __syncthreads();
    T r = smem_warp[warp] + incl - v;
    __syncthreads();
    return r;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T *in, size_t n, uint64_t *sums) {
    __shared__ T sw[8];
    __shared__ T tot;
    size_t base = (size_t)blockIdx.x * kScanTile;
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
        if (i < n) acc += in[i];
    }
    block_exclusive_sum<T>(acc, sw, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = (uint64_t)tot;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const T *in, T *out, size_t n,
                                                                   const uint64_t *offs, T *d_total) {
    __shared__ T sw[8];
    __shared__ T tot;
    size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + k;
        v[k] = i < n ? in[i] : T(0);
        acc += v[k];
    }
    T ex = block_exclusive_sum<T>(acc, sw, &tot);
    T run = (T)offs[blockIdx.x] + ex;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        size_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (d_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *d_total = run;
}

}  // namespace

template <class T>
static void scan_level(const T *in, T *out, size_t n, T *d_total, cudaStream_t s, PrimWorkspace &ws, int depth) {
    if (n == 0) {
        if (d_total) MG_CUDA(cudaMemsetAsync(d_total, 0, sizeof(T), s));
        return;
    }
    size_t tiles = ceil_div(n, kScanTile);
    DBuf<uint64_t> &sums = depth == 0 ? ws.scan_a : depth == 1 ? ws.scan_b : ws.scan_c;
    MG_CHECK(depth < 3, MG_ERR_UNSUPPORTED, "scan: input too large");
    uint64_t *bs = sums.ensure(tiles + 1);
    scan_reduce_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, bs);
    MG_LAUNCH_CHECK();
    if (tiles > 1) scan_level<uint64_t>(bs, bs, tiles, nullptr, s, ws, depth + 1);
    else MG_CUDA(cudaMemsetAsync(bs, 0, sizeof(uint64_t), s));
    scan_down_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, bs, d_total);
    MG_LAUNCH_CHECK();
}

template <class T>
void exclusive_scan(const T *in, T *out, size_t n, T *d_total, cudaStream_t s, PrimWorkspace &ws) {
    scan_level<T>(in, out, n, d_total, s, ws, 0);
}

template void exclusive_scan<uint32_t>(const uint32_t *, uint32_t *, size_t, uint32_t *, cudaStream_t, PrimWorkspace &);
template void exclusive_scan<uint64_t>(const uint64_t *, uint64_t *, size_t, uint64_t *, cudaStream_t, PrimWorkspace &);

// ---------------------------------------------------------------------------
// Radix sort.  Tile = 8 warps x 16 rounds x 32 lanes = 4096 keys; warp w owns
// the contiguous sub-tile [w*512, (w+1)*512), visited round by round in lane
// order, so ranks follow input order (stable).
// ---------------------------------------------------------------------------
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsRounds = 16;
constexpr int kRsTile = kRsThreads * kRsRounds;

__global__ void __launch_bounds__(kRsThreads) rs_hist_kernel(const uint64_t *keys, size_t n, int shift,
                                                               uint32_t *hist, uint32_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    size_t base = (size_t)blockIdx.x * kRsTile;
#pragma unroll 4
    for (int k = 0; k < kRsRounds; k++) {
        size_t i = base + (size_t)k * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: keys are ranked inside the tile (warp
// match_any + per-warp digit counters), staged in shared memory in digit
// order, and written out as contiguous runs per digit (coalesced).
template <class V>
__global__ void __launch_bounds__(kRsThreads) rs_scatter_kernel(const uint64_t *keys, const V *vals,
                                                                  uint64_t *okeys, V *ovals, size_t n, int shift,
                                                                  const uint32_t *offs, uint32_t tiles) {
    constexpr bool HasV = !std::is_same<V, NoVal>::value;
    extern __shared__ __align__(16) unsigned char rs_smem[];
    uint64_t *sk = (uint64_t *)rs_smem;                       // kRsTile keys
    V *sv = (V *)(rs_smem + sizeof(uint64_t) * kRsTile);      // kRsTile values
    __shared__ uint32_t cnt[kRsWarps][256];
    __shared__ uint32_t tstart[256], gofs[256], wsum[kRsWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kRsWarps * 256; d += kRsThreads) (&cnt[0][0])[d] = 0;
    __syncthreads();
    const size_t tile0 = (size_t)blockIdx.x * kRsTile;
    const uint32_t tile_n = (uint32_t)(n - tile0 < (size_t)kRsTile ? n - tile0 : (size_t)kRsTile);
    const uint32_t wbase = (uint32_t)warp * (kRsRounds * 32);
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t k[kRsRounds];
    uint32_t rank[kRsRounds];
    V v[HasV ? kRsRounds : 1];
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        uint32_t li = wbase + r * 32 + lane;
        k[r] = li < tile_n ? keys[tile0 + li] : 0;
        if constexpr (HasV) v[r] = li < tile_n ? vals[tile0 + li] : V();
    }
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        uint32_t li = wbase + r * 32 + lane;
        uint32_t d = li < tile_n ? (uint32_t)((k[r] >> shift) & 0xFF) : 0x100u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = __popc(peers & lt);
        uint32_t run = d < 256 ? cnt[warp][d] : 0;
        rank[r] = run + before;
        __syncwarp();
        if (d < 256 && before == 0) cnt[warp][d] = run + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        // per digit: exclusive prefix over warps, digit total, tile-wide
        // exclusive scan of the totals, global offset of this tile's run
        const int d = threadIdx.x;
        uint32_t acc = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) {
            uint32_t c = cnt[w][d];
            cnt[w][d] = acc;
            acc += c;
        }
        uint32_t incl = acc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        gofs[d] = offs[(size_t)d * tiles + blockIdx.x];
        __syncthreads();
        uint32_t before = 0;
        for (int w = 0; w < warp; w++) before += wsum[w];
        tstart[d] = before + incl - acc;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        uint32_t li = wbase + r * 32 + lane;
        if (li < tile_n) {
            uint32_t d = (uint32_t)((k[r] >> shift) & 0xFF);
            uint32_t pos = tstart[d] + cnt[warp][d] + rank[r];
            sk[pos] = k[r];
            if constexpr (HasV) sv[pos] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tile_n; i += kRsThreads) {
        const uint64_t key = sk[i];
        const uint32_t d = (uint32_t)((key >> shift) & 0xFF);
        const uint32_t pos = gofs[d] + (i - tstart[d]);
        okeys[pos] = key;
        if constexpr (HasV) ovals[pos] = sv[i];
    }
}

}  // namespace

template <class V>
bool radix_sort(uint64_t *keys, V *vals, uint64_t *keys_alt, V *vals_alt, size_t n, int bits,
                cudaStream_t s, PrimWorkspace &ws, int lo_bit) {
    if (n <= 1 || bits <= lo_bit) return false;
    MG_CHECK(n < 0xFFFFFFFFull, MG_ERR_UNSUPPORTED, "radix_sort: more than 2^32-1 keys");
    uint32_t tiles = (uint32_t)ceil_div(n, kRsTile);
    uint32_t *hist = ws.hist.ensure((size_t)tiles * 256 + 1);
    uint64_t *ka = keys, *kb = keys_alt;
    V *va = vals, *vb = vals_alt;
    bool flipped = false;
    const size_t smem = (size_t)kRsTile * (sizeof(uint64_t) + (std::is_same<V, NoVal>::value ? 0 : sizeof(V)));
    MG_CUDA(cudaFuncSetAttribute(rs_scatter_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int shift = lo_bit; shift < bits; shift += 8) {
        rs_hist_kernel<<<tiles, kRsThreads, 0, s>>>(ka, n, shift, hist, tiles);
        MG_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(hist, hist, (size_t)tiles * 256, nullptr, s, ws);
        rs_scatter_kernel<V><<<tiles, kRsThreads, smem, s>>>(ka, va, kb, vb, n, shift, hist, tiles);
        MG_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
        flipped = !flipped;
    }
    return flipped;
}

template bool radix_sort<NoVal>(uint64_t *, NoVal *, uint64_t *, NoVal *, size_t, int, cudaStream_t, PrimWorkspace &,
                                int);
template bool radix_sort<uint32_t>(uint64_t *, uint32_t *, uint64_t *, uint32_t *, size_t, int, cudaStream_t,
                                   PrimWorkspace &, int);
template bool radix_sort<double>(uint64_t *, double *, uint64_t *, double *, size_t, int, cudaStream_t,
                                 PrimWorkspace &, int);

}  // namespace mg
