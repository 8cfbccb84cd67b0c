// 4x4 block statistics (the reference's bench/blockinfo.cpp:96-119) on the
// device.
//
// The reference counts distinct keys of std::map<int,int>:
//   plain:    row/4 * 1000005 + col/4        (blocks of the matrix as is)
//   recorder: row/4 * 1000005 + z/4          (z = position in the row: the
//             DBSR packing of consecutive nonzeros)
// in 32-bit int arithmetic, which wraps for row/4 above 2147 (two's
// complement on the reference's build).  The counts here use the same
// wrapped 32-bit keys, so they equal the reference's even where wrapped keys
// of different blocks collide.  Keys are sorted with the device radix sort
// and the distinct values counted.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

__global__ void blockinfo_keys_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                      const int32_t *__restrict__ colIdx, int32_t *__restrict__ kplain,
                                      int32_t *__restrict__ krec) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nwarps) {
    const int32_t s = rowPtr[r], e = rowPtr[r + 1];
    const uint32_t base = (uint32_t)(r / 4) * 1000005u;
    for (int32_t j = s + lane; j < e; j += 32) {
      kplain[j] = (int32_t)(base + (uint32_t)(colIdx[j] / 4));
      krec[j] = (int32_t)(base + (uint32_t)((j - s) / 4));
    }
  }
}

__global__ void count_distinct_sorted_kernel(const int32_t *__restrict__ k, int64_t n,
                                             unsigned long long *__restrict__ out) {
  __shared__ unsigned long long part[8];
  unsigned long long c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c += (i == 0 || k[i] != k[i - 1]) ? 1ull : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    atomicAdd(out, t);
  }
}

static bsp_status count_distinct(int32_t *keys, int32_t *scratch_vals, int64_t n, int64_t *count, cudaStream_t s) {
  BSP_TRY(radix_sort_pairs(keys, scratch_vals, n, 32, s));
  unsigned long long *d = nullptr;
  BSP_TRY(dalloc(&d, 1, s));
  BSP_CUDA(cudaMemsetAsync(d, 0, sizeof(*d), s));
  int64_t g = ceil_div(n, 256);
  if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
  if (g < 1) g = 1;
  count_distinct_sorted_kernel<<<(unsigned)g, 256, 0, s>>>(keys, n, d);
  BSP_LAUNCH_CHECK();
  unsigned long long h = 0;
  BSP_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  dfree(d, s);
  *count = (int64_t)h;
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_blockinfo(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                    const int32_t *colIdx, int64_t *blocks, int64_t *blocks_recorder,
                                    bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(blocks && blocks_recorder, "null output");
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  BSP_CHECK_ARG(rowPtr && (nnz == 0 || colIdx), "null pointer");
  *blocks = 0;
  *blocks_recorder = 0;
  if (nnz == 0 || rows == 0) return BSP_OK;
  cudaStream_t s = as_stream(stream);
  int32_t *kp = nullptr, *kr = nullptr, *v = nullptr;
  BSP_TRY(dalloc(&kp, (size_t)nnz, s));
  BSP_TRY(dalloc(&kr, (size_t)nnz, s));
  BSP_TRY(dalloc(&v, (size_t)nnz, s));
  int64_t g = ceil_div((int64_t)rows * 32, 256);
  if (g > (int64_t)sm_count() * 32) g = (int64_t)sm_count() * 32;
  blockinfo_keys_kernel<<<(unsigned)g, 256, 0, s>>>(rows, rowPtr, colIdx, kp, kr);
  BSP_LAUNCH_CHECK();
  BSP_TRY(count_distinct(kp, v, nnz, blocks, s));
  BSP_TRY(count_distinct(kr, v, nnz, blocks_recorder, s));
  dfree(kp, s);
  dfree(kr, s);
  dfree(v, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}
