// common.cuh -- shared types, error handling and device helpers of the B200
// Louvain engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/mgagcd.h"

namespace mg {

struct Error : std::runtime_error {
    mg_status status;
    Error(mg_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

#define MG_STR2(x) #x
#define MG_STR(x) MG_STR2(x)
#define MG_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw ::mg::Error(e_ == cudaErrorMemoryAllocation ? MG_ERR_OOM : MG_ERR_CUDA,          \
                              std::string(#call) + ": " + cudaGetErrorString(e_) +                 \
                                  " (" __FILE__ ":" MG_STR(__LINE__) ")");                        \
    } while (0)
#define MG_CHECK(cond, st, msg)                                                                    \
    do {                                                                                           \
        if (!(cond)) throw ::mg::Error((st), (msg));                                               \
    } while (0)
// Every kernel launch of the engine is followed by MG_LAUNCH_CHECK(), which
// also counts the launch (reported per run in mg_summary.kernel_launches).
extern thread_local unsigned long long g_kernel_launches;
#define MG_LAUNCH_CHECK()                 \
    do {                                  \
        ::mg::g_kernel_launches++;        \
        MG_CUDA(cudaGetLastError());      \
    } while (0)

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kNumSMs = 148;

// WK_U32: exact 32-bit integer weights, the storage of every coarsened level
// of an integral graph (each coarsened weight is at most the graph's mass,
// which is below 2^32 for integral graphs): 4 bytes per entry instead of 8.
enum WeightKind { WK_UNIT = 0, WK_F32 = 1, WK_F64 = 2, WK_U32 = 5 };
// Kernel variants: weights stored as f32 / f64 whose values are integral
// accumulate in 32-bit integer table slots, which shared and distributed
// shared memory add natively.
enum { WK_F32I = 3, WK_F64I = 4 };
template <int WK>
constexpr bool kIntg = WK == WK_UNIT || WK == WK_F32I || WK == WK_F64I || WK == WK_U32;

inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline uint32_t pow2_at_least(uint64_t x, uint32_t lo = 16) {
    uint32_t p = lo;
    while (p < x) p <<= 1;
    return p;
}

// ---- device buffers ------------------------------------------------------
// Allocation-failure injection (test hook, mg_test_fail_allocation): when
// armed with n, the n-th device allocation of the library from then on fails
// as out of memory, once.  Process-wide.
bool alloc_fault_due();

// Grow-only device allocation owned by the engine (cudaMalloc on growth only).
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    T *ensure(size_t n) {
        if (n > cap) {
            release();
            size_t want = n < 16 ? 16 : n;
            if (alloc_fault_due()) throw Error(MG_ERR_OOM, "device allocation failed (injected by mg_test_fail_allocation)");
            MG_CUDA(cudaMalloc(&p, want * sizeof(T)));
            cap = want;
        }
        return p;
    }
    T *get() const { return p; }
};

// ---- device helpers ----------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Correctly rounded x / d for a divisor fixed for the whole run, with its
// reciprocal r = RN(1/d) computed once on the host: q0 = RN(x*r) lies within
// one ulp of x/d, the remainder x - q0*d is exact in one fma, and
// RN(q0 + rem*r) is then the correctly rounded quotient (Markstein's
// theorem; J.-M. Muller et al., Handbook of Floating-Point Arithmetic,
// ch. 5).  No intermediate of the gain overflows or underflows.  It keeps the
// arithmetic on the FP64 pipe instead of the special-function unit that a
// divide instruction sequence uses.
__device__ __forceinline__ double div_by(double x, double d, double r) {
    const double q0 = __dmul_rn(x, r);
    const double rem = __fma_rn(-q0, d, x);
    return __fma_rn(rem, r, q0);
}
__device__ __forceinline__ float div_by(float x, float d, float r) {
    const float q0 = __fmul_rn(x, r);
    const float rem = __fmaf_rn(-q0, d, x);
    return __fmaf_rn(rem, r, q0);
}
// exact uint32 -> double with one FP64 subtraction: the bits 0x43300000:x
// encode 2^52 + x
__device__ __forceinline__ double u2d(uint32_t x) {
    return __dsub_rn(__hiloint2double(0x43300000, (int)x), 4503599627370496.0);
}

// Multiplicative hash onto [0, 2^bits)
__device__ __forceinline__ uint32_t hash_slot(uint32_t c, int bits) {
    return (c * 0x9E3779B1u) >> (32 - bits);
}
// Multiplicative hash onto [0, size) for arbitrary size
__device__ __forceinline__ uint32_t hash_range(uint32_t c, uint32_t size) {
    return (uint32_t)(((uint64_t)(c * 0x9E3779B1u) * size) >> 32);
}

// splitmix64 finaliser and the counter-based stream built on it; identical to
// the test oracle's generator so that seeded graphs agree bit for bit.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng_key(uint64_t seed, uint64_t stream) {
    return mix64(seed * 0x2545F4914F6CDD1Dull + stream);
}
__host__ __device__ __forceinline__ uint64_t rng_at(uint64_t key, uint64_t ctr) {
    return mix64(key + ctr * 0x9E3779B97F4A7C15ull);
}
__host__ __device__ __forceinline__ uint32_t uni32(uint32_t x, uint32_t range) {
    return (uint32_t)(((uint64_t)x * range) >> 32);
}

}  // namespace mg
