// bins.cu -- degree binning (histogram, scan, stable scatter).
//
// Bin thresholds follow the reference exactly (src/bin/BIN.cu):
//   scheme 0 (10 bins, local move)       <=2,4,8,16,32,128,512,2048,4094,>4094   (BIN.cu:72-92)
//   scheme 1 (11 bins, coarsen symbolic) <=32,64,...,8192,12288,>12288           (BIN.cu:159-181)
//   scheme 2 (9 bins, coarsen numeric)   <=32,64,...,2048,4095,>4095             (BIN.cu:248-266)
// The reference scatters with atomics (order inside a bin unspecified,
// BIN.cu:298-466); here the scatter ranks by vertex id, so every bin lists
// its members in ascending order.
//
// Scheme 3 is the local-move sweep's own grouping (no reference counterpart;
// the sweep's results do not depend on it): 19 degree classes,
//   class 0: deg <= 1, class c (1..17): 2^(c-1) < deg <= 2^c, class 18: > 2^17,
// so that the kernel shape of each class can be chosen freely (see
// lm_kernels.cuh): classes 0-12 go to the tile / shared-memory hash shapes,
// 13-17 to thread-block clusters of 1-16 CTAs, 18 to the global-table path.
#include "engine.cuh"

namespace mg {

int bin_count(int scheme) { return scheme == 0 ? 10 : scheme == 1 ? 11 : scheme == 2 ? 9 : kSweepClasses; }

namespace {

constexpr int kBinThreads = 1024;

__device__ __forceinline__ int bin_of(int scheme, uint32_t d) {
    if (scheme == 3) {
        if (d <= 1) return 0;
        const int c = 32 - __clz(d - 1);  // ceil(log2 d)
        return c < kSweepClasses - 1 ? c : kSweepClasses - 1;
    }
    if (scheme == 0) {
        if (d <= 32) return d <= 2 ? 0 : d <= 4 ? 1 : d <= 8 ? 2 : d <= 16 ? 3 : 4;
        return d <= 128 ? 5 : d <= 512 ? 6 : d <= 2048 ? 7 : d <= 4094 ? 8 : 9;
    } else if (scheme == 1) {
        if (d <= 512) return d <= 32 ? 0 : d <= 64 ? 1 : d <= 128 ? 2 : d <= 256 ? 3 : 4;
        return d <= 1024 ? 5 : d <= 2048 ? 6 : d <= 4096 ? 7 : d <= 8192 ? 8 : d <= 12288 ? 9 : 10;
    } else {
        if (d <= 512) return d <= 32 ? 0 : d <= 64 ? 1 : d <= 128 ? 2 : d <= 256 ? 3 : 4;
        return d <= 1024 ? 5 : d <= 2048 ? 6 : d <= 4095 ? 7 : 8;
    }
}

// counts[b * blocks + blk] = members of bin b in block blk; max degree
__global__ void __launch_bounds__(kBinThreads) bins_count_kernel(int scheme, int nb, uint32_t n, const uint32_t *off,
                                                                  uint32_t *counts, uint32_t blocks,
                                                                  uint32_t *max_deg) {
    __shared__ uint32_t c[kMaxBins];
    __shared__ uint32_t mx;
    if (threadIdx.x < kMaxBins) c[threadIdx.x] = 0;
    if (threadIdx.x == 0) mx = 0;
    __syncthreads();
    uint32_t i = blockIdx.x * kBinThreads + threadIdx.x;
    uint32_t d = 0;
    int b = -1;
    if (i < n) {
        d = off[i + 1] - off[i];
        b = bin_of(scheme, d);
    }
    uint32_t peers = __match_any_sync(0xffffffffu, (uint32_t)b);
    if (b >= 0 && (__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(&c[b], __popc(peers));
    uint32_t wm = __reduce_max_sync(0xffffffffu, d);
    if ((threadIdx.x & 31) == 0) atomicMax(&mx, wm);
    __syncthreads();
    if (threadIdx.x < (unsigned)nb) counts[(size_t)threadIdx.x * blocks + blockIdx.x] = c[threadIdx.x];
    if (threadIdx.x == 0) atomicMax(max_deg, mx);
}

__global__ void __launch_bounds__(kBinThreads) bins_scatter_kernel(int scheme, uint32_t n, const uint32_t *off,
                                                                    const uint32_t *offs, uint32_t blocks,
                                                                    uint32_t *perm) {
    __shared__ uint32_t wc[32][kMaxBins];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = threadIdx.x; t < 32 * kMaxBins; t += kBinThreads) (&wc[0][0])[t] = 0;
    __syncthreads();
    uint32_t i = blockIdx.x * kBinThreads + threadIdx.x;
    int b = -1;
    if (i < n) b = bin_of(scheme, off[i + 1] - off[i]);
    uint32_t peers = __match_any_sync(0xffffffffu, (uint32_t)b);
    uint32_t before = __popc(peers & ((1u << lane) - 1u));
    if (b >= 0 && before == 0) wc[warp][b] = __popc(peers);
    __syncthreads();
    if (threadIdx.x < kMaxBins) {
        uint32_t acc = 0;
        for (int w = 0; w < 32; w++) {
            uint32_t x = wc[w][threadIdx.x];
            wc[w][threadIdx.x] = acc;
            acc += x;
        }
    }
    __syncthreads();
    if (b >= 0) perm[offs[(size_t)b * blocks + blockIdx.x] + wc[warp][b] + before] = i;
}

}  // namespace

void compute_bins(int scheme, uint32_t n, const uint32_t *d_off, uint32_t *d_perm, Bins &out, cudaStream_t s,
                  PrimWorkspace &ws) {
    MG_CHECK(scheme >= 0 && scheme <= 3, MG_ERR_INVALID, "bins: scheme must be 0, 1, 2 or 3");
    int nb = bin_count(scheme);
    out = Bins();
    out.scheme = scheme;
    out.count = nb;
    if (n == 0) return;
    uint32_t blocks = (uint32_t)ceil_div(n, kBinThreads);
    size_t ncnt = (size_t)nb * blocks;
    // counts | max_degree | total in one allocation
    uint32_t *cnt = ws.bins.ensure(ncnt + 2);
    uint32_t *maxd = cnt + ncnt;
    MG_CUDA(cudaMemsetAsync(maxd, 0, sizeof(uint32_t), s));
    bins_count_kernel<<<blocks, kBinThreads, 0, s>>>(scheme, nb, n, d_off, cnt, blocks, maxd);
    MG_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(cnt, cnt, ncnt, maxd + 1, s, ws);
    bins_scatter_kernel<<<blocks, kBinThreads, 0, s>>>(scheme, n, d_off, cnt, blocks, d_perm);
    MG_LAUNCH_CHECK();
    // bin b starts at cnt[b * blocks]
    std::vector<uint32_t> starts(nb + 2);
    for (int b = 0; b < nb; b++)
        MG_CUDA(cudaMemcpyAsync(&starts[b], cnt + (size_t)b * blocks, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(&starts[nb], maxd, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    out.max_degree = starts[nb];
    uint32_t total = starts[nb + 1];
    for (int b = 0; b < nb; b++) {
        out.offset[b] = starts[b];
        out.size[b] = (b + 1 < nb ? starts[b + 1] : total) - starts[b];
    }
}

}  // namespace mg
