// Error state, small C-ABI utilities and a device exclusive scan used by the
// format conversions (the reference uses thrust::exclusive_scan for the same
// steps: src/amgT.cu:1008,1043,1190 and src/csrspmv.cu:157).
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

// ---------------------------------------------------------------------------
// Exclusive scan of int32 values, three phases (tile sums, scan of the tile
// sums, rescan with offsets).  Each tile is 256 threads x 8 items.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive sum of one int64 per thread: warp shuffle scans, then
// warp 0 scans the per-warp totals.  Returns the block total in `total`.
__device__ __forceinline__ void block_exclusive_sum(int64_t v, int64_t &excl, int64_t &total,
                                                    int64_t *warp_tot /* [kScanThreads/32 + 1] smem */) {
  constexpr int kWarps = kScanThreads / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    const int64_t t = lane < kWarps ? warp_tot[lane] : 0;
    int64_t ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t u = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += u;
    }
    if (lane < kWarps) warp_tot[lane] = ti - t;
    if (lane == kWarps - 1) warp_tot[kWarps] = ti;
  }
  __syncthreads();
  excl = inc - v + warp_tot[w];
  total = warp_tot[kWarps];
  __syncthreads();  // warp_tot may be reused by the caller's next call
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const int32_t *__restrict__ in, int64_t n,
                                                               int64_t *__restrict__ tile_sums) {
  __shared__ int64_t wt[kScanThreads / 32 + 1];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int64_t excl, total;
  block_exclusive_sum(s, excl, total, wt);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of n int64 values in place, one CTA walking the tiles.
__global__ void __launch_bounds__(kScanThreads) scan_i64_single(int64_t *__restrict__ v, int64_t n) {
  __shared__ int64_t wt[kScanThreads / 32 + 1];
  int64_t carry = 0;
  for (int64_t tile = 0; tile < n; tile += kScanTile) {
    const int64_t base = tile + (int64_t)threadIdx.x * kScanItems;
    int64_t items[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      items[k] = base + k < n ? v[base + k] : 0;
      s += items[k];
    }
    int64_t excl, total;
    block_exclusive_sum(s, excl, total, wt);
    excl += carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < n) v[base + k] = excl;
      excl += items[k];
    }
    carry += total;
  }
}

// Rescans each tile with its offset.  in == out is allowed: every thread
// reads its items before writing them.  The grand total goes to *total_out.
__global__ void __launch_bounds__(kScanThreads) scan_rescan(const int32_t *in, int32_t *out, int64_t n,
                                                            const int64_t *__restrict__ tile_off,
                                                            int64_t *__restrict__ total_out, int64_t ntiles) {
  __shared__ int64_t wt[kScanThreads / 32 + 1];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int32_t items[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    items[k] = base + k < n ? in[base + k] : 0;
    s += items[k];
  }
  int64_t excl, total;
  block_exclusive_sum(s, excl, total, wt);
  excl += tile_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = (int32_t)excl;
    excl += items[k];
  }
  if (blockIdx.x == ntiles - 1 && threadIdx.x == kScanThreads - 1 && total_out) *total_out = excl;
}

bsp_status exclusive_scan_i32(const int32_t *in, int32_t *out, int64_t n, int64_t *d_total,
                              cudaStream_t s) {
  if (n <= 0) {
    if (d_total) BSP_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int64_t), s));
    return BSP_OK;
  }
  const int64_t ntiles = ceil_div(n, kScanTile);
  int64_t *tile = nullptr;
  BSP_TRY(dalloc(&tile, ntiles, s));
  scan_tile_sums<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tile);
  BSP_LAUNCH_CHECK();
  scan_i64_single<<<1, kScanThreads, 0, s>>>(tile, ntiles);
  BSP_LAUNCH_CHECK();
  scan_rescan<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, out, n, tile, d_total, ntiles);
  BSP_LAUNCH_CHECK();
  dfree(tile, s);
  return BSP_OK;
}

bsp_status read_i64(const int64_t *d, int64_t *h, cudaStream_t s) {
  BSP_CUDA(cudaMemcpyAsync(h, d, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

bsp_status read_i32(const int32_t *d, int32_t *h, cudaStream_t s) {
  BSP_CUDA(cudaMemcpyAsync(h, d, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" const char *bsp_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *bsp_version(void) { return "libbspmv 0.1 (sm_100a)"; }

extern "C" bsp_status bsp_memcpy_d2h(void *dst_host, const void *src_dev, size_t bytes) {
  clear_error();
  if (bytes == 0) return BSP_OK;
  BSP_CHECK_ARG(dst_host && src_dev, "null pointer");
  BSP_CUDA(cudaMemcpy(dst_host, src_dev, bytes, cudaMemcpyDeviceToHost));
  return BSP_OK;
}

extern "C" bsp_status bsp_memcpy_h2d(void *dst_dev, const void *src_host, size_t bytes) {
  clear_error();
  if (bytes == 0) return BSP_OK;
  BSP_CHECK_ARG(dst_dev && src_host, "null pointer");
  BSP_CUDA(cudaMemcpy(dst_dev, src_host, bytes, cudaMemcpyHostToDevice));
  return BSP_OK;
}

extern "C" bsp_status bsp_device_sync(void) {
  clear_error();
  BSP_CUDA(cudaDeviceSynchronize());
  return BSP_OK;
}

extern "C" bsp_status bsp_device_alloc(void **ptr, size_t bytes) {
  clear_error();
  BSP_CHECK_ARG(ptr, "null pointer");
  *ptr = nullptr;
  if (bytes == 0) return BSP_OK;
  const cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    BSP_FAIL(BSP_ERR_ALLOC, std::string("cudaMalloc(") + std::to_string(bytes) + " B) -> " + cudaGetErrorString(e));
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_device_free(void *ptr) {
  clear_error();
  if (ptr) BSP_CUDA(cudaFree(ptr));
  return BSP_OK;
}

// ---------------------------------------------------------------------------
// Random-gather rate probe (measurement only).  `count` gathers of `width`
// bytes at pseudo-random width-aligned offsets of buf: width 8 is one 8-byte
// load per thread (a DASP / CSR x gather), width 16..256 is width/16 lanes
// each loading 16 bytes of one row (the SpMM B-row gathers).  Eight gathers
// per thread are issued before any is consumed; the loaded words are folded
// into an integer that is stored only if it hits an impossible value, so the
// loads stay.  Read-only path, default caching, as the SpMV/SpMM kernels.
namespace bsp {
__device__ __forceinline__ uint64_t probe_hash(uint64_t z) {
  z ^= z >> 33;
  z *= 0xff51afd7ed558ccdull;
  z ^= z >> 33;
  return z;
}

template <int W>
__global__ void __launch_bounds__(256) gather_probe_kernel(const unsigned char *__restrict__ buf, int64_t nslots,
                                                           int64_t count, uint64_t seed,
                                                           unsigned long long *__restrict__ sink) {
  constexpr int L = W >= 16 ? W / 16 : 1;       // lanes per gather
  constexpr int U = 8;                          // gathers in flight per thread
  const int64_t lane_grp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / L;
  const int sub = threadIdx.x % L;
  const int64_t groups = (int64_t)gridDim.x * blockDim.x / L;
  uint64_t acc = 0;
  for (int64_t g0 = lane_grp * U; g0 < count; g0 += groups * U) {
    uint64_t v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t g = g0 + u;
      const int64_t slot = (int64_t)__umul64hi(probe_hash(seed ^ (uint64_t)g), (uint64_t)nslots);  // < nslots
      if (g < count) {
        if constexpr (W == 8) {
          v[u] = __ldg(reinterpret_cast<const unsigned long long *>(buf) + slot);
        } else {
          const uint4 q = __ldg(reinterpret_cast<const uint4 *>(buf + slot * W) + sub);
          v[u] = (uint64_t)q.x ^ ((uint64_t)q.y << 7) ^ ((uint64_t)q.z << 13) ^ ((uint64_t)q.w << 29);
        }
      } else {
        v[u] = 0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) acc += v[u];
  }
  if (acc == 0x9E3779B97F4A7C15ull) *sink = acc;
}
}  // namespace bsp

extern "C" bsp_status bsp_gather_probe(const void *buf, size_t bytes, int32_t width, int64_t count, uint64_t seed,
                                       void *sink, bsp_stream_t stream) {
  using namespace bsp;
  clear_error();
  BSP_CHECK_ARG(buf && sink && count >= 0, "bad argument");
  BSP_CHECK_ARG(width == 8 || width == 16 || width == 32 || width == 64 || width == 128 || width == 256,
                "width must be 8, 16, 32, 64, 128 or 256 bytes");
  BSP_CHECK_ARG((uintptr_t)buf % 16 == 0 && bytes >= (size_t)width, "buffer must be 16-byte aligned and hold a row");
  const int64_t nslots = (int64_t)(bytes / (size_t)width);
  cudaStream_t s = as_stream(stream);
  int blocks = 0;
  const unsigned grid = (unsigned)sm_count() * 8;
  auto *k = reinterpret_cast<unsigned long long *>(sink);
  const auto *b = static_cast<const unsigned char *>(buf);
  switch (width) {
    case 8: gather_probe_kernel<8><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
    case 16: gather_probe_kernel<16><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
    case 32: gather_probe_kernel<32><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
    case 64: gather_probe_kernel<64><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
    case 128: gather_probe_kernel<128><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
    default: gather_probe_kernel<256><<<grid, 256, 0, s>>>(b, nslots, count, seed, k); break;
  }
  (void)blocks;
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}
