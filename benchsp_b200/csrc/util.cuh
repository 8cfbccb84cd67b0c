// Declarations of the internal device utilities (util.cu).
#pragma once
#include "bsp_internal.cuh"

namespace bsp {
// out[i] = sum(in[0..i)), n items; in == out allowed.  *d_total (device,
// optional) receives sum(in[0..n)).  Allocates tile scratch on `s`.
bsp_status exclusive_scan_i32(const int32_t *in, int32_t *out, int64_t n, int64_t *d_total, cudaStream_t s);
// Synchronous single-value device->host reads on stream s.
bsp_status read_i64(const int64_t *d, int64_t *h, cudaStream_t s);
bsp_status read_i32(const int32_t *d, int32_t *h, cudaStream_t s);
}  // namespace bsp

namespace bsp {
// Stable LSD radix sort (8-bit digits) of int32 (key, value) pairs by key;
// keys must be non-negative and < 2^key_bits.  sort.cu.
bsp_status radix_sort_pairs(int32_t *keys, int32_t *vals, int64_t n, int key_bits, cudaStream_t s);
// Host read of max(v[0..n)) (0 for n == 0; values must be >= 0).
bsp_status max_i32(const int32_t *v, int64_t n, int32_t *h_max, cudaStream_t s);
// Number of bits needed for values in [0, maxv].
int bits_for(int32_t maxv);
}  // namespace bsp
