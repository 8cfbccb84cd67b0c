// Stable LSD radix sort of (key, value) int32 pairs on the device, used by
// the format conversions that reorder rows by length:
//   * DBSR's recorder step sorts rows ascending by length with ties in row
//     order (std::sort of (len, row) pairs, reference include/dbsr.h:209-216);
//   * DASP sorts its row-block rows descending by length, stable
//     (radix_sort/count_sort, reference src/dasp.cu:214-246, :1244).
// A tile is 256 keys, one per thread.  Per pass (8-bit digit): a digit
// histogram per tile, an exclusive scan over the digit-major/tile-minor
// histogram matrix, then a scatter in which every key finds its rank among
// equal digits of its tile with warp match + per-warp counts, so the order
// of equal digits is preserved.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kSortTile = 256;

__global__ void __launch_bounds__(kSortTile) radix_hist_kernel(const int32_t *__restrict__ keys, int64_t n,
                                                               int shift, int64_t ntiles,
                                                               int32_t *__restrict__ hist) {
  __shared__ int32_t cnt[256];
  const int t = threadIdx.x;
  cnt[t] = 0;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kSortTile + t;
  if (i < n) atomicAdd(&cnt[((uint32_t)keys[i] >> shift) & 255u], 1);
  __syncthreads();
  hist[(int64_t)t * ntiles + blockIdx.x] = cnt[t];
}

__global__ void __launch_bounds__(kSortTile) radix_scatter_kernel(const int32_t *__restrict__ kin,
                                                                  const int32_t *__restrict__ vin,
                                                                  int32_t *__restrict__ kout,
                                                                  int32_t *__restrict__ vout, int64_t n, int shift,
                                                                  int64_t ntiles,
                                                                  const int32_t *__restrict__ offs) {
  __shared__ int32_t wcnt[kSortTile / 32][256];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
  for (int k = 0; k < kSortTile / 32; ++k) wcnt[k][t] = 0;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kSortTile + t;
  const bool valid = i < n;
  const int32_t key = valid ? kin[i] : 0;
  const unsigned d = valid ? (((uint32_t)key >> shift) & 255u) : 256u;  // 256 = no digit
  const unsigned peers = __match_any_sync(0xffffffffu, d);
  const int rank = __popc(peers & ((1u << lane) - 1u));
  if (valid && lane == __ffs(peers) - 1) wcnt[w][d] = __popc(peers);
  __syncthreads();
  {  // exclusive prefix over the warps, digit t
    int32_t run = 0;
#pragma unroll
    for (int k = 0; k < kSortTile / 32; ++k) {
      const int32_t c = wcnt[k][t];
      wcnt[k][t] = run;
      run += c;
    }
  }
  __syncthreads();
  if (valid) {
    const int64_t pos = (int64_t)offs[(int64_t)d * ntiles + blockIdx.x] + wcnt[w][d] + rank;
    kout[pos] = key;
    vout[pos] = vin[i];
  }
}

__global__ void max_i32_kernel(const int32_t *__restrict__ v, int64_t n, int32_t *__restrict__ out) {
  int32_t m = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, v[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

bsp_status max_i32(const int32_t *v, int64_t n, int32_t *h_max, cudaStream_t s) {
  int32_t *d = nullptr;
  BSP_TRY(dalloc(&d, 1, s));
  BSP_CUDA(cudaMemsetAsync(d, 0, sizeof(int32_t), s));
  if (n > 0) {
    int64_t blocks = ceil_div(n, 256);
    if (blocks > (int64_t)sm_count() * 16) blocks = (int64_t)sm_count() * 16;
    max_i32_kernel<<<(unsigned)blocks, 256, 0, s>>>(v, n, d);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(read_i32(d, h_max, s));
  dfree(d, s);
  return BSP_OK;
}

bsp_status radix_sort_pairs(int32_t *keys, int32_t *vals, int64_t n, int key_bits, cudaStream_t s) {
  if (n <= 1 || key_bits <= 0) return BSP_OK;
  const int64_t ntiles = ceil_div(n, kSortTile);
  if ((int64_t)256 * ntiles > INT32_MAX) BSP_FAIL(BSP_ERR_UNSUPPORTED, "sort too large");
  int32_t *k2 = nullptr, *v2 = nullptr, *hist = nullptr;
  BSP_TRY(dalloc(&k2, (size_t)n, s));
  BSP_TRY(dalloc(&v2, (size_t)n, s));
  BSP_TRY(dalloc(&hist, (size_t)(256 * ntiles), s));
  int32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += 8, ++passes) {
    radix_hist_kernel<<<(unsigned)ntiles, kSortTile, 0, s>>>(ka, n, shift, ntiles, hist);
    BSP_LAUNCH_CHECK();
    BSP_TRY(exclusive_scan_i32(hist, hist, 256 * ntiles, nullptr, s));
    radix_scatter_kernel<<<(unsigned)ntiles, kSortTile, 0, s>>>(ka, va, kb, vb, n, shift, ntiles, hist);
    BSP_LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (passes & 1) {
    BSP_CUDA(cudaMemcpyAsync(keys, ka, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    BSP_CUDA(cudaMemcpyAsync(vals, va, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
  }
  dfree(k2, s);
  dfree(v2, s);
  dfree(hist, s);
  return BSP_OK;
}

int bits_for(int32_t maxv) {
  int b = 0;
  while (b < 31 && (1ll << b) <= (int64_t)maxv) ++b;
  return b;
}

}  // namespace bsp
