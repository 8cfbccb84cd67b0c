// AmgT-style BSR: device CSR->BSR conversion and BSR SpMV for sm_100a.
//
// Conversion (replaces CSR2BSR_GPU, reference src/amgT.cu:1114-1172, and
// BSR_BALANCED_PREPROCESS_GPU, :1174-1200).  The reference counts block
// columns with a 32,768-column bitmask window per block-row
// (csr2bsr_get_ptr, :585), bins block-rows by length (:646-731) and fills
// each block-row with a shared-memory hash table whose entries are ranked by
// counting smaller keys (csr2bsr_getidx, :733-850).  Its output is the
// canonical BSR: block columns ascending inside a block-row, 4x4 row-major
// values, bitmap bit r*4+c.  Here the same arrays come from a sort-free,
// hash-free formulation that is fully parallel over the nonzeros:
//   1. an element is the block's representative ("canonical") when it is
//      the first of its block column in its own row and no earlier row of
//      the block-row has that block column (binary search in those rows);
//   2. an exclusive scan of the canonical flags over all nonzeros gives
//      blcPtr directly (the block-rows' nonzeros are contiguous in CSR);
//   3. a block's rank inside its block-row is the number of canonical
//      elements with a smaller block column, summed over the block-row's
//      rows with one binary search per row, so every element finds its
//      block without a hash table.
// The result is bit-identical to the reference's for bs = 4 (blcVal,
// blcIdx, blcMap, blcPtr, rowPtrbyWarp, rowIdxbyWarp, warpnum).
//
// SpMV (replaces bsr_spmv_{tc,cc,balanced_tc,balanced_cc}_fp64,
// :160-322 and :464-521).  The reference gives each warp one block-row (or a
// <=64-block chunk) and adds into y with atomicAdd.  Here:
//   * FFMA: a group of LG lanes owns a block-row; 8 lanes cover a 4x4 block
//     (2 doubles each), so a warp-wide load instruction moves 512
//     contiguous bytes; loads of U steps are issued before any FMA; the
//     row sums are reduced with shuffles and y is written once (no atomics).
//   * DMMA: FP64 mma.sync.m8n8k4 on block pairs (the reference's scheme,
//     rows of two blocks stacked into the 8x4 A fragment) with deterministic
//     extraction of the useful diagonal sub-blocks.
#include <algorithm>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kWarpCapacity = 64;  // blocks per balanced chunk (reference include/common.h:7)

// Number of the first element >= key in a[lo, hi).
__device__ __forceinline__ int32_t lower_bound_i32(const int32_t *__restrict__ a, int32_t lo, int32_t hi,
                                                   int32_t key) {
  while (lo < hi) {
    int32_t mid = (lo + hi) >> 1;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Step 1: canonical flags; one warp per row (grid-stride over rows).  Blocks
// are tm x tk: block-row r/tm, block column c/tk.
__global__ void bsr_canonical_kernel(int32_t rows, int32_t tm, int32_t tk, const int32_t *__restrict__ rowPtr,
                                     const int32_t *__restrict__ colIdx, int32_t *__restrict__ flag) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t rr = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rr < rows; rr += nwarps) {
    const int32_t r = (int32_t)rr;
    const int32_t s = rowPtr[r], e = rowPtr[r + 1];
    const int32_t r0 = (r / tm) * tm;
    for (int32_t j = s + lane; j < e; j += 32) {
      const int32_t b = colIdx[j] / tk;
      int32_t canon = (j == s) || (colIdx[j - 1] / tk != b);
      for (int32_t q = r0; q < r && canon; ++q) {
        const int32_t qs = rowPtr[q], qe = rowPtr[q + 1];
        const int32_t p = lower_bound_i32(colIdx, qs, qe, b * tk);
        if (p < qe && colIdx[p] / tk == b) canon = 0;
      }
      flag[j] = canon;
    }
  }
}

// blcPtr[br] = pos[rowPtr[br*tm]]: the block-row's nonzeros are contiguous,
// so the scan of the canonical flags at its first nonzero counts the blocks
// of all earlier block-rows.  pos has nnz+1 entries (pos[nnz] = blc_num).
__global__ void bsr_ptr_kernel(int32_t rows, int32_t blc_row, int32_t tm, const int32_t *__restrict__ rowPtr,
                               const int32_t *__restrict__ pos, int32_t *__restrict__ blcPtr) {
  for (int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; br <= blc_row;
       br += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = br * tm;
    blcPtr[br] = pos[rowPtr[r < rows ? r : rows]];
  }
}

template <typename MapT>
__device__ __forceinline__ void map_or(MapT *map, int64_t blk, int bit);
template <>
__device__ __forceinline__ void map_or<uint16_t>(uint16_t *map, int64_t blk, int bit) {
  // 16-bit maps are OR-ed through the aligned 32-bit word that holds them.
  unsigned *w = reinterpret_cast<unsigned *>(map) + (blk >> 1);
  atomicOr(w, (1u << bit) << ((blk & 1) * 16));
}
template <>
__device__ __forceinline__ void map_or<uint64_t>(uint64_t *map, int64_t blk, int bit) {
  atomicOr(reinterpret_cast<unsigned long long *>(map) + blk, 1ull << bit);
}
template <>
__device__ __forceinline__ void map_or<char>(char *, int64_t, int) {}  // no bitmap for tiles > 64 entries

// Step 3: every nonzero locates its block and scatters value + bitmap bit.
// rank = number of distinct block columns < b in the block-row = sum over the
// block-row's rows q of the canonical elements in q before lower_bound(b*tk).
template <typename MapT>
__global__ void bsr_fill_kernel(int32_t rows, int32_t tm, int32_t tk, const int32_t *__restrict__ rowPtr,
                                const int32_t *__restrict__ colIdx, const double *__restrict__ val,
                                const int32_t *__restrict__ pos, const int32_t *__restrict__ blcPtr,
                                int32_t *__restrict__ blcIdx, double *__restrict__ blcVal, MapT *blcMap) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t rr = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rr < rows; rr += nwarps) {
    const int32_t r = (int32_t)rr;
    const int32_t br = r / tm, r0 = br * tm;
    const int32_t r1 = r0 + tm < rows ? r0 + tm : rows;
    const int32_t s = rowPtr[r], e = rowPtr[r + 1];
    const int32_t base = blcPtr[br], end_blk = blcPtr[br + 1];
    for (int32_t j = s + lane; j < e; j += 32) {
      const int32_t c = colIdx[j];
      const int32_t b = c / tk;
      int32_t rank = 0;
      for (int32_t q = r0; q < r1; ++q) {
        const int32_t qs = rowPtr[q], qe = rowPtr[q + 1];
        const int32_t p = lower_bound_i32(colIdx, qs, qe, b * tk);
        rank += pos[p] - pos[qs];
      }
      const int64_t blk = (int64_t)base + rank;
      if (blk >= end_blk) continue;  // only reachable for unsorted input
      const int in_r = r - r0, in_c = c - b * tk;
      blcVal[blk * tm * tk + in_r * tk + in_c] = val[j];
      map_or<MapT>(blcMap, blk, in_r * tk + in_c);
      blcIdx[blk] = b;
    }
  }
}

__global__ void bsr_chunks_kernel(int32_t blc_row, const int32_t *__restrict__ blcPtr, int32_t *__restrict__ cnt,
                                  double avg_len, double *__restrict__ sq) {
  // cnt[br] = ceil(len/64) (get_rowPtrbyWarp, amgT.cu:523); sq[br] = (len-avg)^2.
  for (int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; br < blc_row;
       br += (int64_t)gridDim.x * blockDim.x) {
    const int32_t len = blcPtr[br + 1] - blcPtr[br];
    cnt[br] = (len + kWarpCapacity - 1) / kWarpCapacity;
    const double d = (double)len - avg_len;
    sq[br] = d * d;
  }
}

__global__ void bsr_rowidx_kernel(int32_t blc_row, const int32_t *__restrict__ rowPtrbyWarp,
                                  int32_t *__restrict__ rowIdxbyWarp) {
  for (int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; br < blc_row;
       br += (int64_t)gridDim.x * blockDim.x)
    for (int32_t w = rowPtrbyWarp[br]; w < rowPtrbyWarp[br + 1]; ++w) rowIdxbyWarp[w] = (int32_t)br;
}

// Deterministic sum of doubles (single CTA, fixed order per thread then a
// fixed tree), for the block-length standard deviation.
__global__ void sum_f64_kernel(const double *__restrict__ v, int64_t n, double *__restrict__ out) {
  __shared__ double part[256];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 256) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = part[0];
}

__global__ void count_full_blocks_kernel(int64_t nb, int bs, const void *map, int32_t *out) {
  __shared__ int32_t part[256];
  int32_t c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
    if (bs == 4)
      c += reinterpret_cast<const uint16_t *>(map)[i] == 0xffffu;
    else
      c += reinterpret_cast<const uint64_t *>(map)[i] == ~0ull;
  }
  part[threadIdx.x] = c;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, part[0]);
}

static unsigned grid_for(int64_t n, int threads) {
  int64_t b = ceil_div(n, threads);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

static unsigned grid_for(int64_t n, int threads);

// Canonical tm x tk blocking of a CSR matrix (block columns ascending per
// block-row, row-major values).  map16 (tm*tk <= 16) or map64 (<= 64) get the
// occupancy bitmaps when non-null.  Outputs are allocated here.
bsp_status csr2blocks(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx, const double *values,
                      int32_t tm, int32_t tk, int32_t *blc_num_out, int32_t **blcPtr, int32_t **blcIdx,
                      double **blcVal, uint16_t **map16, uint64_t **map64, cudaStream_t s) {
  const int32_t blc_row = (int32_t)ceil_div(rows, tm);
  int32_t *pos = nullptr;
  int64_t *d_total = nullptr;
  BSP_TRY(dalloc(&pos, (size_t)nnz + 1, s));
  BSP_TRY(dalloc(&d_total, 2, s));
  BSP_CUDA(cudaMemsetAsync(pos + nnz, 0, sizeof(int32_t), s));
  if (nnz > 0) {
    bsr_canonical_kernel<<<grid_for((int64_t)rows * 32, 256), 256, 0, s>>>(rows, tm, tk, rowPtr, colIdx, pos);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(pos, pos, (int64_t)nnz + 1, d_total, s));
  int64_t total = 0;
  BSP_TRY(read_i64(d_total, &total, s));
  dfree(d_total, s);
  if (total > INT32_MAX / ((int64_t)tm * tk)) BSP_FAIL(BSP_ERR_UNSUPPORTED, "too many blocks for int32 indexing");
  const int32_t nb = (int32_t)total;
  *blc_num_out = nb;
  BSP_TRY(dalloc(blcPtr, (size_t)blc_row + 1, s));
  bsr_ptr_kernel<<<grid_for((int64_t)blc_row + 1, 256), 256, 0, s>>>(rows, blc_row, tm, rowPtr, pos, *blcPtr);
  BSP_LAUNCH_CHECK();
  BSP_TRY(dalloc(blcIdx, (size_t)nb, s));
  BSP_TRY(dalloc(blcVal, (size_t)nb * tm * tk, s));
  BSP_CUDA(cudaMemsetAsync(*blcVal, 0, sizeof(double) * (size_t)nb * tm * tk, s));
  const unsigned g = grid_for((int64_t)rows * 32, 256);
  if (map16) {
    // blc_num + 1 entries as the reference allocates (amgT.cu:1162), rounded
    // up to whole 32-bit words for the word-wide OR.
    const size_t n16 = ((size_t)nb + 2) & ~size_t(1);
    BSP_TRY(dalloc(map16, n16, s));
    BSP_CUDA(cudaMemsetAsync(*map16, 0, sizeof(uint16_t) * n16, s));
    if (nnz > 0)
      bsr_fill_kernel<uint16_t><<<g, 256, 0, s>>>(rows, tm, tk, rowPtr, colIdx, values, pos, *blcPtr, *blcIdx,
                                                  *blcVal, *map16);
  } else if (map64) {
    BSP_TRY(dalloc(map64, (size_t)nb + 1, s));
    BSP_CUDA(cudaMemsetAsync(*map64, 0, sizeof(uint64_t) * ((size_t)nb + 1), s));
    if (nnz > 0)
      bsr_fill_kernel<uint64_t><<<g, 256, 0, s>>>(rows, tm, tk, rowPtr, colIdx, values, pos, *blcPtr, *blcIdx,
                                                  *blcVal, *map64);
  } else if (nnz > 0) {
    bsr_fill_kernel<char><<<g, 256, 0, s>>>(rows, tm, tk, rowPtr, colIdx, values, pos, *blcPtr, *blcIdx, *blcVal,
                                            nullptr);
  }
  BSP_LAUNCH_CHECK();
  dfree(pos, s);
  return BSP_OK;
}

bsp_status csr2bsr_impl(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                        const double *values, int32_t bs, bsp_bsr *out, cudaStream_t s) {
  bsp_bsr m{};
  m.row = rows;
  m.col = cols;
  m.bs = bs;
  m.blc_row = (int32_t)ceil_div(rows, bs);
  m.blc_col = (int32_t)ceil_div(cols, bs);
  m.true_nnz = nnz;
  uint16_t *m16 = nullptr;
  uint64_t *m64 = nullptr;
  BSP_TRY(csr2blocks(rows, nnz, rowPtr, colIdx, values, bs, bs, &m.blc_num, &m.blcPtr, &m.blcIdx, &m.blcVal,
                     bs == 4 ? &m16 : nullptr, bs == 4 ? nullptr : &m64, s));
  m.blcMap = bs == 4 ? (void *)m16 : (void *)m64;
  m.nnz = m.blc_num * bs * bs;
  m.avg_nnz = m.blc_num > 0 ? (double)nnz / (double)m.blc_num : 0.0;
  int64_t *d_total = nullptr;
  BSP_TRY(dalloc(&d_total, 1, s));

  // Balanced chunks and block-length statistics.
  double *sq = nullptr, *d_sum = nullptr;
  BSP_TRY(dalloc(&m.rowPtrbyWarp, (size_t)m.blc_row + 1, s));
  BSP_TRY(dalloc(&sq, (size_t)m.blc_row + 1, s));
  BSP_TRY(dalloc(&d_sum, 1, s));
  const double avg_len = m.blc_row > 0 ? (double)m.blc_num / (double)m.blc_row : 0.0;
  BSP_CUDA(cudaMemsetAsync(m.rowPtrbyWarp, 0, sizeof(int32_t) * ((size_t)m.blc_row + 1), s));
  if (m.blc_row > 0) {
    bsr_chunks_kernel<<<grid_for(m.blc_row, 256), 256, 0, s>>>(m.blc_row, m.blcPtr, m.rowPtrbyWarp, avg_len, sq);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(m.rowPtrbyWarp, m.rowPtrbyWarp, (int64_t)m.blc_row + 1, d_total, s));
  int64_t warpnum = 0;
  BSP_TRY(read_i64(d_total, &warpnum, s));
  m.warpnum = (int32_t)warpnum;
  BSP_TRY(dalloc(&m.rowIdxbyWarp, (size_t)m.warpnum, s));
  if (m.blc_row > 0) {
    bsr_rowidx_kernel<<<grid_for(m.blc_row, 256), 256, 0, s>>>(m.blc_row, m.rowPtrbyWarp, m.rowIdxbyWarp);
    BSP_LAUNCH_CHECK();
    sum_f64_kernel<<<1, 256, 0, s>>>(sq, m.blc_row, d_sum);
    BSP_LAUNCH_CHECK();
    double ss = 0.0;
    BSP_CUDA(cudaMemcpyAsync(&ss, d_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
    BSP_CUDA(cudaStreamSynchronize(s));
    // The reference takes a single-precision square root (amgT.cu:1155).
    m.stand = (double)sqrtf((float)(ss / m.blc_row));
  }
  int32_t *d_full = nullptr;
  BSP_TRY(dalloc(&d_full, 1, s));
  BSP_CUDA(cudaMemsetAsync(d_full, 0, sizeof(int32_t), s));
  if (m.blc_num > 0) {
    count_full_blocks_kernel<<<grid_for(m.blc_num, 256), 256, 0, s>>>(m.blc_num, bs, m.blcMap, d_full);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(read_i32(d_full, &m.dense_blocks, s));
  dfree(d_full, s);
  dfree(sq, s);
  dfree(d_sum, s);
  dfree(d_total, s);
  *out = m;
  return BSP_OK;
}

// ---------------------------------------------------------------------------
// FFMA SpMV.  Every lane streams 4 consecutive block values (one 256-bit
// load) and the matching 4 entries of x.  BS = block size (4 or 8); LPB =
// BS*BS/4 lanes per block; LG lanes per block-row (a multiple of LPB); U =
// block steps whose loads are issued before the FMAs; XV4 = x is 32-byte
// aligned so its 4 entries come in one load.
template <int BS, int LG, int U, bool XV4, bool PF>
__global__ void __launch_bounds__(256) bsr_ffma_kernel(int32_t blc_row, int32_t row, int32_t col,
                                                       const int32_t *__restrict__ blcPtr,
                                                       const int32_t *__restrict__ blcIdx,
                                                       const double *__restrict__ blcVal,
                                                       const double *__restrict__ x, double *__restrict__ y,
                                                       double alpha, double beta) {
  constexpr int LPB = BS * BS / 4;  // lanes per block
  constexpr int BPS = LG / LPB;     // blocks per step
  static_assert(LG % LPB == 0 && LG <= 32, "bad lane group");
  const int lane = threadIdx.x & 31;
  const int gl = lane & (LG - 1);  // lane inside the group
  const int slot = gl / LPB;       // which block of the step
  const int e = gl % LPB;          // 4-value chunk inside the block
  const int r = (4 * e) / BS;      // block row this lane accumulates
  const int c = (4 * e) % BS;      // first of its four columns
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / LG);
  const int64_t warp_first = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LG;
  for (int64_t base = warp_first; base < blc_row; base += groups) {
    const int64_t br = base + lane / LG;
    const bool active = br < blc_row;
    const int32_t s = active ? blcPtr[br] : 0;
    const int32_t t = active ? blcPtr[br + 1] : 0;
    double acc0 = 0.0, acc1 = 0.0;
    for (int32_t k0 = s; k0 < t; k0 += BPS * U) {
      f64x4 v[U];
      f64x4 xv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t blk = k0 + u * BPS + slot;
        if (blk < t) {
          v[u] = PF ? ld_stream_f64x4_pf(blcVal + (int64_t)blk * (BS * BS) + 4 * e)
                    : ld_stream_f64x4(blcVal + (int64_t)blk * (BS * BS) + 4 * e);
          const int64_t xc = (int64_t)__ldg(&blcIdx[blk]) * BS + c;
          const double *xp = x + xc;
          if (XV4 && xc + 4 <= col) {
            xv[u] = ld_x4(xp);
          } else {
            // unaligned x, or the last block column running past the end of x
            xv[u].x = xc < col ? ld_x(xp) : 0.0;
            xv[u].y = xc + 1 < col ? ld_x(xp + 1) : 0.0;
            xv[u].z = xc + 2 < col ? ld_x(xp + 2) : 0.0;
            xv[u].w = xc + 3 < col ? ld_x(xp + 3) : 0.0;
          }
        } else {
          v[u] = f64x4{0.0, 0.0, 0.0, 0.0};
          xv[u] = f64x4{0.0, 0.0, 0.0, 0.0};
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        acc0 = fma(v[u].x, xv[u].x, acc0);
        acc1 = fma(v[u].y, xv[u].y, acc1);
        acc0 = fma(v[u].z, xv[u].z, acc0);
        acc1 = fma(v[u].w, xv[u].w, acc1);
      }
    }
    double acc = acc0 + acc1;
    // Lanes of the same block row r: the BS/4 lanes inside a block, then the
    // BPS block slots of the group.
#pragma unroll
    for (int o = 1; o < BS / 4; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
#pragma unroll
    for (int o = LPB; o < LG; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (active && slot == 0 && (e % (BS / 4)) == 0) {
      const int64_t yi = br * BS + r;
      if (yi < row) {
        double res = alpha * acc;
        if (beta != 0.0) res += beta * y[yi];
        y[yi] = res;
      }
    }
  }
}

__device__ __forceinline__ void dmma_m8n8k4(double &c0, double &c1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// DMMA SpMV for 4x4 blocks: one warp per block-row, two blocks per MMA.
// A (8x4) = the two row-major blocks stacked (lane l holds A[l/4][l%4] =
// blcVal[16*i + l]); B (4x8) column n<4 holds x of block i, n>=4 x of block
// i+1 (lane l holds B[l%4][l/4]).  C[r][0] accumulates block i's row r and
// C[4+r][4] block i+1's row r; y_r = C[r][0] + C[4+r][4].
__global__ void __launch_bounds__(256) bsr4_dmma_kernel(int32_t blc_row, int32_t row, int32_t col,
                                                        const int32_t *__restrict__ blcPtr,
                                                        const int32_t *__restrict__ blcIdx,
                                                        const double *__restrict__ blcVal,
                                                        const double *__restrict__ x, double *__restrict__ y,
                                                        double alpha, double beta) {
  const int lane = threadIdx.x & 31;
  const uint64_t pol = evict_first_policy();
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t br = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; br < blc_row; br += nwarps) {
    const int32_t s = blcPtr[br], t = blcPtr[br + 1];
    double c0 = 0.0, c1 = 0.0;
    const int half = lane >> 4;
    for (int32_t i = s; i < t; i += 2) {
      const bool valid = (i + half) < t;
      double a = 0.0, b = 0.0;
      if (valid) {
        a = ld_stream_f64(blcVal + (int64_t)i * 16 + lane, pol);
        const int64_t xc = (int64_t)__ldg(&blcIdx[i + half]) * 4 + (lane & 3);
        b = xc < col ? ld_x(x + xc) : 0.0;
      }
      dmma_m8n8k4(c0, c1, a, b);
    }
    const double other = __shfl_down_sync(0xffffffffu, c0, 18);
    if (lane < 16 && (lane & 3) == 0) {
      const int64_t yi = br * 4 + (lane >> 2);
      if (yi < row) {
        double res = alpha * (c0 + other);
        if (beta != 0.0) res += beta * y[yi];
        y[yi] = res;
      }
    }
  }
}

template <int BS, int LG, int U, bool PF>
static bsp_status launch_ffma(const bsp_bsr *m, const double *x, double *y, double a, double b, int64_t max_blocks,
                              cudaStream_t s) {
  const int threads = 256;
  int64_t blocks = ceil_div(m->blc_row, threads / LG);
  const int64_t cap = max_blocks > 0 ? max_blocks : (int64_t)sm_count() * 64;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  if (((uintptr_t)x & 31) == 0)
    bsr_ffma_kernel<BS, LG, U, true, PF><<<(unsigned)blocks, threads, 0, s>>>(
        m->blc_row, m->row, m->col, m->blcPtr, m->blcIdx, m->blcVal, x, y, a, b);
  else
    bsr_ffma_kernel<BS, LG, U, false, PF><<<(unsigned)blocks, threads, 0, s>>>(
        m->blc_row, m->row, m->col, m->blcPtr, m->blcIdx, m->blcVal, x, y, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

using FfmaLauncher = bsp_status (*)(const bsp_bsr *, const double *, double *, double, double, int64_t,
                                    cudaStream_t);

// Variant table: (bs, lanes per block-row, unroll, L2 256-byte hint).
struct FfmaVariant {
  int bs, lanes, unroll, pf;
  FfmaLauncher fn;
};
#define BSP_FV(BS, LG, U, PF) {BS, LG, U, PF, &launch_ffma<BS, LG, U, PF != 0>}
static const FfmaVariant kFfmaVariants[] = {
    BSP_FV(4, 4, 1, 0),  BSP_FV(4, 4, 2, 0),  BSP_FV(4, 4, 4, 0),  BSP_FV(4, 8, 1, 0),  BSP_FV(4, 8, 2, 0),
    BSP_FV(4, 8, 4, 0),  BSP_FV(4, 16, 1, 0), BSP_FV(4, 16, 2, 0), BSP_FV(4, 16, 4, 0), BSP_FV(4, 32, 1, 0),
    BSP_FV(4, 32, 2, 0), BSP_FV(4, 32, 4, 0), BSP_FV(4, 4, 1, 1),  BSP_FV(4, 8, 1, 1),  BSP_FV(4, 16, 1, 1),
    BSP_FV(4, 32, 1, 1), BSP_FV(4, 16, 2, 1), BSP_FV(8, 16, 1, 0), BSP_FV(8, 16, 2, 0), BSP_FV(8, 16, 4, 0),
    BSP_FV(8, 32, 1, 0), BSP_FV(8, 32, 2, 0), BSP_FV(8, 32, 4, 0), BSP_FV(8, 16, 1, 1), BSP_FV(8, 32, 1, 1),
};
#undef BSP_FV

static const FfmaVariant *find_ffma(int bs, int lanes, int unroll, int pf) {
  for (const FfmaVariant &v : kFfmaVariants)
    if (v.bs == bs && v.lanes == lanes && v.unroll == unroll && v.pf == pf) return &v;
  return nullptr;
}

// Default variant from the mean blocks per block-row.  One block step per
// loop trip (unroll 1) keeps registers low enough for full occupancy, which
// measured faster than deeper unrolling on B200 (27-point 4x4 stencil:
// 135 us at unroll 1 against 159 us at 2 and 216 us at 4, 16 lanes).
static const FfmaVariant *default_ffma(const bsp_bsr *m) {
  const double avg_len = (double)m->blc_num / (double)m->blc_row;
  if (m->bs == 8) return avg_len > 4.0 ? find_ffma(8, 32, 1, 0) : find_ffma(8, 16, 1, 0);
  if (avg_len > 12.0) return find_ffma(4, 16, 1, 0);
  if (avg_len > 4.0) return find_ffma(4, 8, 1, 0);
  return find_ffma(4, 4, 1, 0);
}

bsp_status bsr_spmv_impl(const bsp_bsr *m, const double *x, double *y, double alpha, double beta, int32_t algo,
                         cudaStream_t s) {
  if (m->blc_row == 0) return BSP_OK;
  // 256-bit value loads need 32-byte aligned blocks (library allocations are).
  if (((uintptr_t)m->blcVal & 31) != 0) BSP_FAIL(BSP_ERR_INVALID, "blcVal must be 32-byte aligned");
  if (algo == BSP_BSR_AUTO) algo = BSP_BSR_FFMA;
  if (algo == BSP_BSR_ADAPTIVE) algo = (m->bs == 4 && m->avg_nnz >= 10.0) ? BSP_BSR_DMMA : BSP_BSR_FFMA;
  if (algo == BSP_BSR_DMMA) {
    if (m->bs != 4) BSP_FAIL(BSP_ERR_UNSUPPORTED, "DMMA path is for 4x4 blocks");
    int64_t blocks = ceil_div(m->blc_row, 8);
    const int64_t cap = (int64_t)sm_count() * 64;
    if (blocks > cap) blocks = cap;
    bsr4_dmma_kernel<<<(unsigned)blocks, 256, 0, s>>>(m->blc_row, m->row, m->col, m->blcPtr, m->blcIdx, m->blcVal, x,
                                                      y, alpha, beta);
    BSP_LAUNCH_CHECK();
    return BSP_OK;
  }
  if (algo != BSP_BSR_FFMA) BSP_FAIL(BSP_ERR_INVALID, "unknown BSR algo");
  if (m->bs != 4 && m->bs != 8) BSP_FAIL(BSP_ERR_UNSUPPORTED, "block size must be 4 or 8");
  return default_ffma(m)->fn(m, x, y, alpha, beta, 0, s);
}

// FFMA SpMV of block rows [lo, hi) only (y given for the whole matrix), with
// the kernel shape chosen for the whole matrix.
// Block rows [lo, hi) (the host-buffer plan's ranges); max_blocks > 0 caps
// the grid (the kernel strides over its block rows).
bsp_status bsr_spmv_rows(const bsp_bsr *m, int32_t lo, int32_t hi, const double *x, double *y, double alpha,
                         double beta, int64_t max_blocks, cudaStream_t s) {
  if (hi <= lo) return BSP_OK;
  if (((uintptr_t)m->blcVal & 31) != 0) BSP_FAIL(BSP_ERR_INVALID, "blcVal must be 32-byte aligned");
  bsp_bsr sub = *m;
  sub.blcPtr = m->blcPtr + lo;  // block offsets stay absolute
  sub.blc_row = hi - lo;
  sub.row = std::min<int64_t>((int64_t)m->row - (int64_t)lo * m->bs, (int64_t)(hi - lo) * m->bs);
  return default_ffma(m)->fn(&sub, x, y + (int64_t)lo * m->bs, alpha, beta, max_blocks, s);
}

bsp_status bsr_spmv_variant(const bsp_bsr *m, const double *x, double *y, double alpha, double beta, int lanes,
                            int unroll, int pf, cudaStream_t s) {
  if (m->blc_row == 0) return BSP_OK;
  if (((uintptr_t)m->blcVal & 31) != 0) BSP_FAIL(BSP_ERR_INVALID, "blcVal must be 32-byte aligned");
  const FfmaVariant *v = find_ffma(m->bs, lanes, unroll, pf);
  if (!v) BSP_FAIL(BSP_ERR_UNSUPPORTED, "no FFMA variant with these lanes/unroll/prefetch");
  return v->fn(m, x, y, alpha, beta, 0, s);
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_csr2bsr(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                  const int32_t *colIdx, const double *values, int32_t bs, bsp_bsr *out,
                                  bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out, "null output descriptor");
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  BSP_CHECK_ARG(bs == 4 || bs == 8, "block size must be 4 or 8");
  BSP_CHECK_ARG(rowPtr && (nnz == 0 || (colIdx && values)), "null pointer");
  return csr2bsr_impl(rows, cols, nnz, rowPtr, colIdx, values, bs, out, as_stream(stream));
}

extern "C" bsp_status bsp_bsr_free(bsp_bsr *m) {
  clear_error();
  if (!m) return BSP_OK;
  cudaStream_t s = 0;
  dfree(m->blcPtr, s);
  dfree(m->blcIdx, s);
  dfree(m->blcVal, s);
  if (m->blcMap) cudaFreeAsync(m->blcMap, s);
  m->blcMap = nullptr;
  dfree(m->rowPtrbyWarp, s);
  dfree(m->rowIdxbyWarp, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_spmv(const bsp_bsr *m, const double *x, double *y, double alpha, double beta,
                                   int32_t algo, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && x && y, "null pointer");
  BSP_CHECK_ARG(m->bs == 4 || m->bs == 8, "block size must be 4 or 8");
  return bsr_spmv_impl(m, x, y, alpha, beta, algo, as_stream(stream));
}

extern "C" bsp_status bsp_bsr_spmv_host(const bsp_bsr *m, const double *x_host, double *y_host, double alpha,
                                        double beta, int32_t algo, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && x_host && y_host, "null pointer");
  BSP_CHECK_ARG(m->bs == 4 || m->bs == 8, "block size must be 4 or 8");
  cudaStream_t s = as_stream(stream);
  double *dx = nullptr, *dy = nullptr;
  BSP_TRY(dalloc(&dx, (size_t)m->col, s));
  bsp_status st = dalloc(&dy, (size_t)m->row, s);
  if (st != BSP_OK) {
    dfree(dx, s);
    return st;
  }
  cudaError_t e = cudaMemcpyAsync(dx, x_host, sizeof(double) * m->col, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && beta != 0.0)
    e = cudaMemcpyAsync(dy, y_host, sizeof(double) * m->row, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    st = bsr_spmv_impl(m, dx, dy, alpha, beta, algo, s);
    if (st == BSP_OK) e = cudaMemcpyAsync(y_host, dy, sizeof(double) * m->row, cudaMemcpyDeviceToHost, s);
  }
  dfree(dx, s);
  dfree(dy, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) BSP_FAIL(BSP_ERR_CUDA, cudaGetErrorString(e));
  return st;
}

extern "C" bsp_status bsp_bsr_spmv_variant(const bsp_bsr *m, const double *x, double *y, double alpha,
                                           double beta, int32_t lanes_per_blockrow, int32_t unroll,
                                           int32_t l2_prefetch, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && x && y, "null pointer");
  return bsr_spmv_variant(m, x, y, alpha, beta, lanes_per_blockrow, unroll, l2_prefetch, as_stream(stream));
}
