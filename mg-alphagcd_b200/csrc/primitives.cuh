// primitives.cuh -- device-wide scan and LSD radix sort, hand-written for
// sm_100a (used by coarsening, graph construction and the heavy-vertex
// table layout).
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"

namespace mg {

struct NoVal {};

// Scratch owned by a caller and reused across calls (grow-only).
struct PrimWorkspace {
    DBuf<uint64_t> scan_a, scan_b, scan_c;  // block sums of the scan levels
    DBuf<uint32_t> hist;                    // radix tile histograms
    DBuf<uint32_t> bins;                    // degree-bin block counts
};

// out[i] = sum_{j<i} in[i]; returns nothing (the total, when asked for, is
// written to *d_total on the device).  in and out may alias.  T: uint32_t or
// uint64_t.
template <class T>
void exclusive_scan(const T *in, T *out, size_t n, T *d_total, cudaStream_t s, PrimWorkspace &ws);

// Stable LSD radix sort of keys[0,n) on bits [lo_bit, bits) (bits <= 64),
// with an optional payload: keys equal on those bits keep their input order.
// keys/vals and keys_alt/vals_alt are ping-pong buffers of n entries; returns
// true when the result ended in the *_alt buffers.  V: NoVal, uint32_t or
// double.
template <class V>
bool radix_sort(uint64_t *keys, V *vals, uint64_t *keys_alt, V *vals_alt, size_t n, int bits,
                cudaStream_t s, PrimWorkspace &ws, int lo_bit = 0);

// Number of bits needed to represent values < n (at least 1).
inline int bits_for(uint64_t n) {
    int b = 1;
    while (b < 64 && (1ull << b) < n) b++;
    return b;
}

}  // namespace mg
