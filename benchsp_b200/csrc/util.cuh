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
