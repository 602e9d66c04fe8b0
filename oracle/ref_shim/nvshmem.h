/* Single-PE stand-in for the NVSHMEM API surface that MG-alphaGCD uses
 * (oracle test infrastructure only).  With one PE every one-sided get/put
 * is a local load/store, every collective over the world team is the
 * identity, and the symmetric heap is ordinary device memory.  Collective
 * kernel launches become cooperative launches, which is what NVSHMEM does
 * underneath.  Allocations carry 256 bytes of zeroed slack. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#define NVSHMEMX_SUCCESS 0
#define NVSHMEM_TEAM_WORLD 0
#define NVSHMEMX_INIT_WITH_MPI_COMM 0
typedef int nvshmem_team_t;
typedef struct { void *mpi_comm; } nvshmemx_init_attr_t;

static inline int nvshmemx_init_attr(unsigned int, nvshmemx_init_attr_t *) { return 0; }
static inline void nvshmem_finalize(void) {}
static inline int nvshmem_n_pes(void) { return 1; }
static inline int nvshmem_my_pe(void) { return 0; }
static inline void *nvshmem_malloc(size_t n) {
    void *p = nullptr;
    if (cudaMalloc(&p, n + 256) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, n + 256);
    return p;
}
static inline void nvshmem_free(void *p) { if (p) cudaFree(p); }
/* host: wait for the device; device (one PE): nothing to wait for */
static inline __host__ __device__ void nvshmem_barrier_all(void) {
#ifndef __CUDA_ARCH__
    cudaDeviceSynchronize();
#endif
}
static inline void nvshmemx_barrier_all_on_stream(cudaStream_t) {}

static inline int nvshmemx_collective_launch(const void *func, dim3 grid, dim3 block, void **args,
                                             size_t smem, cudaStream_t stream) {
    return cudaLaunchCooperativeKernel(func, grid, block, args, smem, stream) == cudaSuccess ? 0 : 1;
}
static inline int nvshmemx_collective_launch_query_gridsize(const void *func, dim3 block, void **,
                                                            size_t smem, int *grid) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, (int)(block.x * block.y * block.z), smem) != cudaSuccess)
        return 1;
    *grid = per_sm * sms;
    return 0;
}

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t nvshmem_uint32_g(const uint32_t *p, int) { return *p; }
__device__ __forceinline__ double nvshmem_double_g(const double *p, int) { return *p; }
__device__ __forceinline__ long long nvshmem_longlong_g(const long long *p, int) { return *p; }
__host__ __device__ __forceinline__ void nvshmem_uint32_p(uint32_t *p, uint32_t v, int) {
#ifdef __CUDA_ARCH__
    *p = v;
#else
    cudaMemcpy(p, &v, sizeof v, cudaMemcpyHostToDevice);
#endif
}
__device__ __forceinline__ long long nvshmem_longlong_atomic_compare_swap(long long *p, long long cond, long long v, int) {
    return (long long)atomicCAS((unsigned long long *)p, (unsigned long long)cond, (unsigned long long)v);
}
__device__ __forceinline__ int nvshmemx_double_sum_reduce_warp(nvshmem_team_t, double *dst, const double *src, size_t n) {
    if (dst != src) for (size_t i = threadIdx.x % 32; i < n; i += 32) dst[i] = src[i];
    __syncwarp();
    return 0;
}
__device__ __forceinline__ void nvshmemx_double_get_warp(double *dst, const double *src, size_t n, int) {
    for (size_t i = threadIdx.x % 32; i < n; i += 32) dst[i] = src[i];
    __syncwarp();
}
__device__ __forceinline__ void nvshmemx_uint32_put_block(uint32_t *dst, const uint32_t *src, size_t n, int) {
    __syncthreads();
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}
#endif
