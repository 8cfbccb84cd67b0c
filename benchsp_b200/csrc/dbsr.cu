// DBSR ("denser" 4x4 blocks) on the device: conversion and SpMV.
//
// Format (dbsrMat, reference include/matrixFormat.hpp:86-106; built by
// csrTodbsr, include/dbsr.h:10-92): rows are taken four at a time; the z-th
// nonzero of row i goes to block blcPtr[i/4] + z/4 at position
// (i%4)*4 + z%4, so a block holds four consecutive nonzeros of each of four
// rows with one column index per element (padding: column 0, value 0).
// blcPtr counts, per row quad, the largest ceil(len/4).  With the recorder
// step (csrTodbsrWithRecorder, :208-253) rows are first sorted ascending by
// length, ties by row index, and recorderMap[new] = old.  balanceDbsr
// (:94-168) then packs block-rows into warps of <= 64 blocks (prefix,
// warpnum).  Every array here is bit-identical to the reference's.
//
// balanceDbsr's second walk starts from the first walk's leftover fill and
// does not reload the fill after opening a warp (:139-155), so for many
// inputs it pushes block-rows past the warp vector its first walk sized
// (undefined behaviour in the reference).  Here the walk is replayed
// exactly; when it runs past, the warp list simply grows (warpnum = last
// warp + 1) and `balance_overflow` is set, so no block-row is dropped.  When
// the reference stays in bounds the output is identical.
//
// SpMV: the reference kernels (amgT.cu:324-461) overwrite the gathered x
// with 1.0 (fragB = 1.0, :356 and :425) and so return row sums; this kernel
// computes A*x.  Four lanes share a block, each streams one block row (four
// values in one 256-bit load, four column indices in one 128-bit load) and
// gathers its four x entries; padding is masked with the block bitmap.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kDbsrWarpCap = 64;  // WARP_CAPACITY, reference include/common.h:7

__global__ void row_len_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, int32_t *__restrict__ len,
                               int32_t *__restrict__ idx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    len[i] = rowPtr[i + 1] - rowPtr[i];
    idx[i] = (int32_t)i;
  }
}

// New row lengths in sorted order are the sorted keys themselves; gather the
// rows' columns and values (one warp per row).
__global__ void gather_rows_kernel(int32_t rows, const int32_t *__restrict__ order,
                                   const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
                                   const double *__restrict__ val, const int32_t *__restrict__ newPtr,
                                   int32_t *__restrict__ newCol, double *__restrict__ newVal) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < rows; k += nwarps) {
    const int32_t old = order[k];
    const int32_t s = rowPtr[old], e = rowPtr[old + 1], d = newPtr[k];
    for (int32_t j = s + lane; j < e; j += 32) {
      newCol[d + (j - s)] = colIdx[j];
      newVal[d + (j - s)] = val[j];
    }
  }
}

// cnt[b] = max over the quad's rows of ceil(len/4) (dbsr.h:18-23).
__global__ void dbsr_quad_kernel(int32_t rows, int32_t brow, const int32_t *__restrict__ rowPtr,
                                 int32_t *__restrict__ cnt) {
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < brow; b += (int64_t)gridDim.x * blockDim.x) {
    int32_t m = 0;
    for (int64_t i = b * 4; i < b * 4 + 4 && i < rows; ++i) m = max(m, (rowPtr[i + 1] - rowPtr[i] + 3) / 4);
    cnt[b] = m;
  }
}

// Scatter of every nonzero into its block (dbsr.h:65-79); one warp per row.
__global__ void dbsr_fill_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                 const int32_t *__restrict__ colIdx, const double *__restrict__ val,
                                 const int32_t *__restrict__ blcPtr, int32_t *__restrict__ outCol,
                                 double *__restrict__ outVal, uint16_t *__restrict__ map) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < rows; i += nwarps) {
    const int32_t s = rowPtr[i], e = rowPtr[i + 1];
    const int64_t base = blcPtr[i / 4];
    const int rin = (int)(i % 4);
    for (int32_t j = s + lane; j < e; j += 32) {
      const int32_t z = j - s;
      const int64_t blk = base + z / 4;
      const int pos = rin * 4 + z % 4;
      outVal[blk * 16 + pos] = val[j];
      outCol[blk * 16 + pos] = colIdx[j];
      atomicOr(reinterpret_cast<unsigned *>(map) + (blk >> 1), (1u << pos) << ((blk & 1) * 16));
    }
  }
}

// The two greedy walks of balanceDbsr (dbsr.h:94-168), replayed exactly by one
// thread (the walk is a sequential state machine; blc_row iterations, no
// waits).  counts[w] = block-rows pushed to warp w.
__global__ void dbsr_balance_kernel(int32_t brow, const int32_t *__restrict__ blcPtr, int32_t cap_warps,
                                    int32_t *__restrict__ counts, int32_t *__restrict__ info) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t now = 0, warpcount = 0;
  for (int32_t i = 0; i < brow; ++i) {
    const int32_t len = blcPtr[i + 1] - blcPtr[i];
    if (now + len <= kDbsrWarpCap) {
      now += len;
    } else {
      if (now != 0) {
        warpcount++;
        now = 0;
      }
      if (len <= kDbsrWarpCap)
        now = len;
      else
        warpcount += (len + kDbsrWarpCap - 1) / kDbsrWarpCap;
    }
  }
  if (now) warpcount++;
  // second walk: starts from the first walk's leftover `now` (dbsr.h:134-155)
  int32_t now_warp = 0, last = -1, overflow = 0;
  for (int32_t i = 0; i < brow; ++i) {
    const int32_t len = blcPtr[i + 1] - blcPtr[i];
    if (now + len <= kDbsrWarpCap) {
      if (now_warp < cap_warps) counts[now_warp]++;
      last = max(last, now_warp);
      now += len;
    } else {
      if (now != 0) now = 0;
      if (len <= kDbsrWarpCap) {
        now_warp++;
        if (now_warp < cap_warps) counts[now_warp]++;
        last = max(last, now_warp);
      } else {
        for (int32_t j = 1; j <= (len + kDbsrWarpCap - 1) / kDbsrWarpCap; ++j) {
          now_warp++;
          if (now_warp < cap_warps) counts[now_warp]++;
          last = max(last, now_warp);
        }
      }
    }
  }
  if (last >= warpcount) overflow = 1;
  info[0] = warpcount;
  info[1] = overflow ? last + 1 : warpcount;
  info[2] = overflow;
}

static unsigned grid_for_rows(int64_t n, int per_block) {
  int64_t b = ceil_div(n, per_block);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

bsp_status csr2dbsr_impl(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                         const double *values, int32_t recorder, bsp_dbsr *out, cudaStream_t s) {
  bsp_dbsr m{};
  m.row = rows;
  m.col = cols;
  m.nnz = nnz;
  m.blc_row = (rows + 3) / 4;
  m.blc_col = (cols + 3) / 4;
  const int32_t *rp = rowPtr;
  const int32_t *ci = colIdx;
  const double *va = values;
  int32_t *rp2 = nullptr, *ci2 = nullptr, *keys = nullptr;
  double *va2 = nullptr;
  if (recorder && rows > 0) {
    BSP_TRY(dalloc(&keys, (size_t)rows, s));
    BSP_TRY(dalloc(&m.recorderMap, (size_t)rows, s));
    row_len_kernel<<<grid_for_rows(rows, 256), 256, 0, s>>>(rows, rowPtr, keys, m.recorderMap);
    BSP_LAUNCH_CHECK();
    int32_t maxlen = 0;
    BSP_TRY(max_i32(keys, rows, &maxlen, s));
    // std::sort of (len, row) pairs == stable sort by len
    BSP_TRY(radix_sort_pairs(keys, m.recorderMap, rows, bits_for(maxlen), s));
    BSP_TRY(dalloc(&rp2, (size_t)rows + 1, s));
    BSP_CUDA(cudaMemcpyAsync(rp2, keys, sizeof(int32_t) * rows, cudaMemcpyDeviceToDevice, s));
    BSP_CUDA(cudaMemsetAsync(rp2 + rows, 0, sizeof(int32_t), s));
    BSP_TRY(exclusive_scan_i32(rp2, rp2, (int64_t)rows + 1, nullptr, s));
    BSP_TRY(dalloc(&ci2, (size_t)nnz, s));
    BSP_TRY(dalloc(&va2, (size_t)nnz, s));
    gather_rows_kernel<<<grid_for_rows((int64_t)rows * 32, 256), 256, 0, s>>>(rows, m.recorderMap, rowPtr, colIdx,
                                                                             values, rp2, ci2, va2);
    BSP_LAUNCH_CHECK();
    dfree(keys, s);
    rp = rp2;
    ci = ci2;
    va = va2;
  }
  int64_t *d_total = nullptr;
  BSP_TRY(dalloc(&d_total, 1, s));
  BSP_TRY(dalloc(&m.blcPtr, (size_t)m.blc_row + 1, s));
  BSP_CUDA(cudaMemsetAsync(m.blcPtr, 0, sizeof(int32_t) * ((size_t)m.blc_row + 1), s));
  if (m.blc_row > 0) {
    dbsr_quad_kernel<<<grid_for_rows(m.blc_row, 256), 256, 0, s>>>(rows, m.blc_row, rp, m.blcPtr);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(m.blcPtr, m.blcPtr, (int64_t)m.blc_row + 1, d_total, s));
  int64_t total_block = 0;
  BSP_TRY(read_i64(d_total, &total_block, s));
  if (total_block * 16 > INT32_MAX) BSP_FAIL(BSP_ERR_UNSUPPORTED, "too many blocks for int32 indexing");
  m.blc_num = (int32_t)total_block;
  m.blocknnz = (int32_t)(total_block * 16);
  m.avg_nnz = total_block > 0 ? (double)nnz / (double)total_block : 0.0;
  BSP_TRY(dalloc(&m.colIdx, (size_t)m.blocknnz, s));
  BSP_TRY(dalloc(&m.blcVal, (size_t)m.blocknnz, s));
  const size_t map_n = ((size_t)total_block + 2) & ~size_t(1);
  BSP_TRY(dalloc(&m.blcMap, map_n, s));
  BSP_CUDA(cudaMemsetAsync(m.colIdx, 0, sizeof(int32_t) * (size_t)m.blocknnz, s));
  BSP_CUDA(cudaMemsetAsync(m.blcVal, 0, sizeof(double) * (size_t)m.blocknnz, s));
  BSP_CUDA(cudaMemsetAsync(m.blcMap, 0, sizeof(uint16_t) * map_n, s));
  if (rows > 0 && nnz > 0) {
    dbsr_fill_kernel<<<grid_for_rows((int64_t)rows * 32, 256), 256, 0, s>>>(rows, rp, ci, va, m.blcPtr, m.colIdx,
                                                                           m.blcVal, m.blcMap);
    BSP_LAUNCH_CHECK();
  }
  // balanceDbsr: warps <= blc_row + total_block/64 + 1 (each block-row adds at
  // most ceil(len/64) <= len/64 + 1 warps).
  const int64_t cap_warps = (int64_t)m.blc_row + total_block / kDbsrWarpCap + 2;
  int32_t *counts = nullptr, *info = nullptr;
  BSP_TRY(dalloc(&counts, (size_t)cap_warps + 1, s));
  BSP_TRY(dalloc(&info, 4, s));
  BSP_CUDA(cudaMemsetAsync(counts, 0, sizeof(int32_t) * ((size_t)cap_warps + 1), s));
  dbsr_balance_kernel<<<1, 32, 0, s>>>(m.blc_row, m.blcPtr, (int32_t)cap_warps, counts, info);
  BSP_LAUNCH_CHECK();
  int32_t h_info[4] = {0, 0, 0, 0};
  BSP_CUDA(cudaMemcpyAsync(h_info, info, sizeof(h_info), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  m.warpnum = h_info[1];
  m.balance_overflow = h_info[2];
  BSP_TRY(dalloc(&m.prefix, (size_t)m.warpnum + 1, s));
  // prefix = exclusive scan of counts[0..warpnum], counts[warpnum] == 0
  BSP_CUDA(cudaMemsetAsync(counts + m.warpnum, 0, sizeof(int32_t), s));
  BSP_TRY(exclusive_scan_i32(counts, m.prefix, (int64_t)m.warpnum + 1, nullptr, s));
  dfree(counts, s);
  dfree(info, s);
  dfree(d_total, s);
  dfree(rp2, s);
  dfree(ci2, s);
  dfree(va2, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  *out = m;
  return BSP_OK;
}

// LG lanes per block-row (4 lanes per block, LG/4 blocks per step).
template <int LG>
__global__ void __launch_bounds__(256) dbsr_spmv_kernel(int32_t blc_row, int32_t row,
                                                        const int32_t *__restrict__ blcPtr,
                                                        const int32_t *__restrict__ colIdx,
                                                        const double *__restrict__ blcVal,
                                                        const uint16_t *__restrict__ map,
                                                        const int32_t *__restrict__ outIdx,
                                                        const double *__restrict__ x, double *__restrict__ y,
                                                        double alpha, double beta) {
  constexpr int BPS = LG / 4;
  const int lane = threadIdx.x & 31;
  const int gl = lane & (LG - 1);
  const int slot = gl >> 2;
  const int r = gl & 3;
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / LG);
  const int64_t warp_first = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LG;
  for (int64_t base = warp_first; base < blc_row; base += groups) {
    const int64_t br = base + lane / LG;
    const bool active = br < blc_row;
    const int32_t s = active ? blcPtr[br] : 0;
    const int32_t t = active ? blcPtr[br + 1] : 0;
    double acc0 = 0.0, acc1 = 0.0;
    for (int32_t blk = s + slot; blk < t; blk += BPS) {
      const f64x4 v = ld_stream_f64x4(blcVal + (int64_t)blk * 16 + 4 * r);
      const int4 c = __ldg(reinterpret_cast<const int4 *>(colIdx + (int64_t)blk * 16 + 4 * r));
      const unsigned m = (__ldg(&map[blk]) >> (4 * r)) & 15u;
      if (m & 1u) acc0 = fma(v.x, ld_x(x + c.x), acc0);
      if (m & 2u) acc1 = fma(v.y, ld_x(x + c.y), acc1);
      if (m & 4u) acc0 = fma(v.z, ld_x(x + c.z), acc0);
      if (m & 8u) acc1 = fma(v.w, ld_x(x + c.w), acc1);
    }
    double acc = acc0 + acc1;
#pragma unroll
    for (int o = 4; o < LG; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (active && slot == 0) {
      const int64_t pr = br * 4 + r;  // row in the (possibly reordered) DBSR numbering
      if (pr < row) {
        const int64_t yi = outIdx ? outIdx[pr] : pr;
        double res = alpha * acc;
        if (beta != 0.0) res += beta * y[yi];
        y[yi] = res;
      }
    }
  }
}

bsp_status dbsr_spmv_impl(const bsp_dbsr *m, const double *x, double *y, double alpha, double beta,
                          int32_t permuted_output, cudaStream_t s) {
  if (m->blc_row == 0) return BSP_OK;
  if (((uintptr_t)m->blcVal & 31) || ((uintptr_t)m->colIdx & 15))
    BSP_FAIL(BSP_ERR_INVALID, "DBSR arrays must be 32/16-byte aligned");
  const int32_t *outIdx = (permuted_output || !m->recorderMap) ? nullptr : m->recorderMap;
  const double avg = (double)m->blc_num / (double)m->blc_row;
  const int threads = 256;
  auto launch = [&](auto lg_tag) -> bsp_status {
    constexpr int LG = decltype(lg_tag)::value;
    int64_t blocks = ceil_div(m->blc_row, threads / LG);
    const int64_t cap = (int64_t)sm_count() * 64;
    if (blocks > cap) blocks = cap;
    dbsr_spmv_kernel<LG><<<(unsigned)blocks, threads, 0, s>>>(m->blc_row, m->row, m->blcPtr, m->colIdx, m->blcVal,
                                                               m->blcMap, outIdx, x, y, alpha, beta);
    BSP_LAUNCH_CHECK();
    return BSP_OK;
  };
  if (avg > 12.0) return launch(std::integral_constant<int, 16>());
  if (avg > 4.0) return launch(std::integral_constant<int, 8>());
  return launch(std::integral_constant<int, 4>());
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_csr2dbsr(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                   const int32_t *colIdx, const double *values, int32_t recorder, bsp_dbsr *out,
                                   bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out, "null output descriptor");
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  BSP_CHECK_ARG(rowPtr && (nnz == 0 || (colIdx && values)), "null pointer");
  return csr2dbsr_impl(rows, cols, nnz, rowPtr, colIdx, values, recorder, out, as_stream(stream));
}

extern "C" bsp_status bsp_dbsr_free(bsp_dbsr *m) {
  clear_error();
  if (!m) return BSP_OK;
  cudaStream_t s = 0;
  dfree(m->blcPtr, s);
  dfree(m->colIdx, s);
  dfree(m->blcVal, s);
  dfree(m->blcMap, s);
  dfree(m->recorderMap, s);
  dfree(m->prefix, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_dbsr_spmv(const bsp_dbsr *m, const double *x, double *y, double alpha, double beta,
                                    int32_t permuted_output, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && x && y, "null pointer");
  return dbsr_spmv_impl(m, x, y, alpha, beta, permuted_output, as_stream(stream));
}
