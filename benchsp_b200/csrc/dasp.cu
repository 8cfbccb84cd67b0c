// DASP on the device: packing and a single-launch SpMV.
//
// Packing reproduces the host code of the reference's spmv_all
// (src/dasp.cu:827-1482) array for array:
//   * rows are classified by length: 1, 2, 3, 4, 0, long (>= block_longest)
//     and "row-block" (everything else) (:827-859, :876-918);
//   * len-1 and len-3 rows are paired into 8x4 tiles when
//     min(#1, #3)/8 >= 16 (:922-933, :968-988); the rest of the short rows
//     fill 8x4 tiles of 3/4-length rows (:990-1021) and 2&2 tiles holding
//     16 len-2 rows (:1023-1038), each section padded to whole
//     thread-blocks of tiles (:945-955);
//   * long rows are cut into 64-value warp chunks (:1326-1369);
//   * row-block rows are sorted descending by length, stably (radix_sort,
//     :214-246, :1244); every 8-row block keeps 8x4 tiles while a tile is at
//     least `threshold` full (:1382-1413); what is left of each row is the
//     irregular CSR tail (:1424-1436); the regular part is re-laid tile by
//     tile (:1440-1482);
//   * order_rid maps every y slot back to its row (:1289-1306).
// Each step is a data-parallel kernel (classification by a stable radix
// sort on a 3-bit class key, scans for every pointer array, scatter
// kernels for the tiles).  The superX / short_cid_new / short3_* arrays that
// spmv_all builds and uploads are never read by its kernel (:1045-1239,
// :1311-1327) and are not built.
//
// SpMV: the reference launches dasp_spmv2 then longPart_sum and extracts the
// diagonal of FP64 mma.sync.m8n8k4 products (1/8 of the MMA output is used).
// Here one launch covers every part with CUDA-core FP64 FMA (the path is
// bandwidth- and gather-bound; tiles are read as whole 32-byte rows where
// alignment allows, and each thread issues all its loads before its x
// gathers).  Long rows: a warp takes a group of up to 4 of the row's 64-value
// chunks, publishes its partial with a release increment of the row's
// counter, and the warp that completes the count sums the row's partials in
// group order and resets the counter (no waiting), so the result is
// deterministic.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kTile = 32;          // MMA_M * MMA_K
constexpr int kLongChunk = 64;     // MMA_M * MMA_K * loopNum_long
constexpr int kLongGroup = 4;      // chunks of one long row per SpMV warp
enum : int32_t { kC1 = 0, kC2 = 1, kC3 = 2, kC4 = 3, kCLong = 4, kCBlock = 5, kCZero = 6 };

__global__ void dasp_classify_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, int32_t block_longest,
                                     int32_t *__restrict__ key, int32_t *__restrict__ idx,
                                     int32_t *__restrict__ counts) {
  __shared__ int32_t c[8];
  if (threadIdx.x < 8) c[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t len = rowPtr[i + 1] - rowPtr[i];
    // the reference's test order: 1, 3, 2, 0, 4, long, block (dasp.cu:830-858)
    int32_t k;
    if (len == 1)
      k = kC1;
    else if (len == 3)
      k = kC3;
    else if (len == 2)
      k = kC2;
    else if (len == 0)
      k = kCZero;
    else if (len == 4)
      k = kC4;
    else if (len >= block_longest)
      k = kCLong;
    else
      k = kCBlock;
    key[i] = k;
    idx[i] = (int32_t)i;
    atomicAdd(&c[k], 1);
  }
  __syncthreads();
  if (threadIdx.x < 7 && c[threadIdx.x]) atomicAdd(&counts[threadIdx.x], c[threadIdx.x]);
}

struct DaspShortLayout {
  int32_t s1, s2, s3, s4, common13;  // s1/s3 after the 1&3 pairing
  const int32_t *rid1, *rid2, *rid3, *rid4;
  int32_t f13, f34;                  // fill0_nnz_short13 / 34
};

// One thread per short-part item: the s1 single rows, the common13 1&3 pairs,
// the remaining len-3 rows, the len-4 rows, then the len-2 rows.
__global__ void dasp_short_fill_kernel(DaspShortLayout L, const int32_t *__restrict__ rowPtr,
                                       const int32_t *__restrict__ colIdx, const double *__restrict__ val,
                                       double *__restrict__ sval, int32_t *__restrict__ scid) {
  const int64_t total = (int64_t)L.s1 + L.common13 + L.s3 + L.s4 + L.s2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = q;
    if (t < L.s1) {  // dasp.cu:961-966
      const int32_t s = rowPtr[L.rid1[t]];
      sval[t] = val[s];
      scid[t] = colIdx[s];
      continue;
    }
    t -= L.s1;
    if (t < L.common13) {  // dasp.cu:968-988
      const int64_t i = t / 8, j = t % 8;
      const int64_t o = L.s1 + i * kTile + j * 4;
      const int32_t a = rowPtr[L.rid1[L.s1 + t]];
      const int32_t b = rowPtr[L.rid3[t]];
      sval[o] = val[a];
      scid[o] = colIdx[a];
      for (int k = 0; k < 3; ++k) {
        sval[o + 1 + k] = val[b + k];
        scid[o + 1 + k] = colIdx[b + k];
      }
      continue;
    }
    t -= L.common13;
    if (t < L.s3) {  // dasp.cu:990-1005
      const int64_t o = L.s1 + L.f13 + t * 4;
      const int32_t b = rowPtr[L.rid3[L.common13 + t]];
      for (int k = 0; k < 3; ++k) {
        sval[o + k] = val[b + k];
        scid[o + k] = colIdx[b + k];
      }
      continue;
    }
    t -= L.s3;
    if (t < L.s4) {  // dasp.cu:1007-1021
      const int64_t o = L.s1 + L.f13 + ((int64_t)L.s3 + t) * 4;
      const int32_t b = rowPtr[L.rid4[t]];
      for (int k = 0; k < 4; ++k) {
        sval[o + k] = val[b + k];
        scid[o + k] = colIdx[b + k];
      }
      continue;
    }
    t -= L.s4;
    {  // len-2 rows, 16 per 8x4 tile (dasp.cu:1023-1038)
      const int64_t i = t / 16, j = t % 16;
      const int64_t o = L.s1 + L.f13 + L.f34 + i * kTile + (j % 8) * 4 + (j / 8) * 2;
      const int32_t b = rowPtr[L.rid2[t]];
      sval[o] = val[b];
      sval[o + 1] = val[b + 1];
      scid[o] = colIdx[b];
      scid[o + 1] = colIdx[b + 1];
    }
  }
}

__global__ void dasp_long_count_kernel(int32_t row_long, const int32_t *__restrict__ lrid,
                                       const int32_t *__restrict__ rowPtr, int32_t *__restrict__ nwarp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row_long; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t len = rowPtr[lrid[i] + 1] - rowPtr[lrid[i]];
    nwarp[i] = (len + kLongChunk - 1) / kLongChunk;
  }
}

// Copies each long row to long_ptr_warp[i]*64 (dasp.cu:1346-1369) and tags
// its warps with the long-row index.
__global__ void dasp_long_fill_kernel(int32_t row_long, const int32_t *__restrict__ lrid,
                                      const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
                                      const double *__restrict__ val, const int32_t *__restrict__ wptr,
                                      double *__restrict__ lval, int32_t *__restrict__ lcid,
                                      int32_t *__restrict__ wrow) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < row_long; i += nwarps) {
    const int32_t s = rowPtr[lrid[i]], e = rowPtr[lrid[i] + 1];
    const int64_t o = (int64_t)wptr[i] * kLongChunk;
    for (int32_t j = s + lane; j < e; j += 32) {
      lval[o + (j - s)] = val[j];
      lcid[o + (j - s)] = colIdx[j];
    }
    for (int32_t w = wptr[i] + lane; w < wptr[i + 1]; w += 32) wrow[w] = (int32_t)i;
  }
}

__global__ void dasp_long_groups_kernel(int32_t row_long, const int32_t *__restrict__ wptr,
                                        int32_t *__restrict__ ngroups) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row_long; i += (int64_t)gridDim.x * blockDim.x)
    ngroups[i] = (wptr[i + 1] - wptr[i] + kLongGroup - 1) / kLongGroup;
}

__global__ void dasp_group_info_kernel(int32_t row_long, const int32_t *__restrict__ gptr,
                                       const int32_t *__restrict__ wptr, int4 *__restrict__ info) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < row_long; i += nwarps) {
    const int32_t g0 = gptr[i], ng = gptr[i + 1] - g0;
    for (int32_t k = lane; k < ng; k += 32) {
      const int32_t c0 = wptr[i] + k * kLongGroup;
      const int32_t nc = min(kLongGroup, wptr[i + 1] - c0);
      info[g0 + k] = make_int4((int32_t)i, c0, g0, nc | (ng << 4));
    }
  }
}

__global__ void dasp_block_keys_kernel(int32_t row_block, const int32_t *__restrict__ ridA,
                                       const int32_t *__restrict__ rowPtr, int32_t block_longest,
                                       int32_t *__restrict__ key, int32_t *__restrict__ val) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row_block; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = ridA[i];
    key[i] = block_longest - 1 - (rowPtr[r + 1] - rowPtr[r]);  // ascending key = descending length
    val[i] = r;
  }
}

__global__ void dasp_sorted_len_kernel(int32_t row_block, const int32_t *__restrict__ key, int32_t block_longest,
                                       int32_t *__restrict__ len) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= row_block; i += (int64_t)gridDim.x * blockDim.x)
    len[i] = i < row_block ? block_longest - 1 - key[i] : 0;
}

// Tiles kept per 8-row block and the irregular tail of each row
// (dasp.cu:1382-1413).  rpt = prefix of the sorted lengths.
__global__ void dasp_block_fill_kernel(int32_t blocknum, int32_t row_block, const int32_t *__restrict__ rpt,
                                       double threshold, int32_t *__restrict__ blockPtr,
                                       int32_t *__restrict__ irreg) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < blocknum; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rs = i * 8;
    const int64_t re = (i + 1) * 8 >= row_block ? row_block : (i + 1) * 8;
    int32_t k = 1;
    while (true) {
      int32_t block_nnz = 0;
      for (int64_t r = rs; r < re; ++r) {
        const int32_t len = rpt[r + 1] - rpt[r];
        if (len / 4 >= k)
          block_nnz += 4;
        else if (len / 4 == k - 1)
          block_nnz += len % 4;
      }
      if (block_nnz >= threshold * 4 * 8) {
        blockPtr[i] += 32;
      } else {
        for (int64_t r = rs; r < re; ++r) {
          const int32_t len = rpt[r + 1] - rpt[r];
          irreg[r] = len - (k - 1) * 4 > 0 ? len - (k - 1) * 4 : 0;
        }
        break;
      }
      ++k;
    }
  }
}

// Irregular tail: the last irreg_len nonzeros of each sorted row
// (dasp.cu:1424-1436); one warp per row.
__global__ void dasp_irreg_fill_kernel(int32_t row_block, const int32_t *__restrict__ sortedA,
                                       const int32_t *__restrict__ irpt, const int32_t *__restrict__ rowPtr,
                                       const int32_t *__restrict__ colIdx, const double *__restrict__ val,
                                       double *__restrict__ ival, int32_t *__restrict__ icid) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < row_block; i += nwarps) {
    const int32_t o = irpt[i], n = irpt[i + 1] - o;
    const int32_t end = rowPtr[sortedA[i] + 1];
    for (int32_t j = lane; j < n; j += 32) {
      ival[o + j] = val[end - n + j];
      icid[o + j] = colIdx[end - n + j];
    }
  }
}

// Regular tiles (dasp.cu:1440-1482): element o of block bid is tile
// t = f/32, row r = (f%32)/4, column c = f%4 of the block (f = o -
// blockPtr[bid]) and holds entry 4t+c of sorted row 8*bid+r (0 past the row).
__global__ void dasp_reg_fill_kernel(int64_t total, int32_t blocknum, int32_t row_block,
                                     const int32_t *__restrict__ blockPtr, const int32_t *__restrict__ sortedA,
                                     const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
                                     const double *__restrict__ val, double *__restrict__ rval,
                                     int32_t *__restrict__ rcid) {
  for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += (int64_t)gridDim.x * blockDim.x) {
    int32_t lo = 0, hi = blocknum;  // last bid with blockPtr[bid] <= o
    while (hi - lo > 1) {
      const int32_t mid = (lo + hi) >> 1;
      if (blockPtr[mid] <= o)
        lo = mid;
      else
        hi = mid;
    }
    const int32_t bid = lo;
    const int64_t f = o - blockPtr[bid];
    const int64_t t = f / kTile, r = (f % kTile) / 4, c = f % 4;
    const int64_t i = t * 4 + c;
    const int64_t row = (int64_t)bid * 8 + r;
    double v = 0.0;
    int32_t cc = 0;
    if (row < row_block) {
      const int32_t s = rowPtr[sortedA[row]], e = rowPtr[sortedA[row] + 1];
      if (i < e - s) {
        v = val[s + i];
        cc = colIdx[s + i];
      }
    }
    rval[o] = v;
    rcid[o] = cc;
  }
}

struct DaspOrder {
  int32_t row_long, row_block, s1, common13, s3, s4, s2, row_zero;
  const int32_t *lrid, *sortedA, *rid1, *rid3, *rid4, *rid2, *zrid;
};

__global__ void dasp_order_kernel(DaspOrder O, int32_t *__restrict__ order) {
  const int64_t total = (int64_t)O.row_long + O.row_block + O.s1 + 2 * (int64_t)O.common13 + O.s3 + O.s4 + O.s2 +
                        O.row_zero;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = k;
    int32_t r;
    if (t < O.row_long) {
      r = O.lrid[t];
    } else if ((t -= O.row_long) < O.row_block) {
      r = O.sortedA[t];
    } else if ((t -= O.row_block) < O.s1) {
      r = O.rid1[t];
    } else if ((t -= O.s1) < 2 * (int64_t)O.common13) {
      const int64_t i = t / 16, j = t % 16;  // 8 len-1 rows then 8 len-3 rows per tile (:1294-1303)
      r = j < 8 ? O.rid1[O.s1 + i * 8 + j] : O.rid3[i * 8 + (j - 8)];
    } else if ((t -= 2 * (int64_t)O.common13) < O.s3) {
      r = O.rid3[O.common13 + t];
    } else if ((t -= O.s3) < O.s4) {
      r = O.rid4[t];
    } else if ((t -= O.s4) < O.s2) {
      r = O.rid2[t];
    } else {
      r = O.zrid[t - O.s2];
    }
    order[k] = r;
  }
}

static unsigned dgrid(int64_t n, int per_block = 256) {
  int64_t b = ceil_div(n, per_block);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

bsp_status csr2dasp_impl(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                         const double *values, double threshold, int32_t block_longest, bsp_dasp *out,
                         cudaStream_t s) {
  bsp_dasp d{};
  d.rows = rows;
  d.cols = cols;
  d.nnz = nnz;
  d.threshold = threshold;
  d.block_longest = block_longest;
  // --- classification: stable partition by class (row order kept inside)
  int32_t *key = nullptr, *sorted = nullptr, *cnt = nullptr;
  BSP_TRY(dalloc(&key, (size_t)rows + 1, s));
  BSP_TRY(dalloc(&sorted, (size_t)rows + 1, s));
  BSP_TRY(dalloc(&cnt, 8, s));
  BSP_CUDA(cudaMemsetAsync(cnt, 0, 8 * sizeof(int32_t), s));
  if (rows > 0) {
    dasp_classify_kernel<<<dgrid(rows), 256, 0, s>>>(rows, rowPtr, block_longest, key, sorted, cnt);
    BSP_LAUNCH_CHECK();
    BSP_TRY(radix_sort_pairs(key, sorted, rows, 3, s));
  }
  int32_t c[8];
  BSP_CUDA(cudaMemcpyAsync(c, cnt, sizeof(c), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  const int32_t s1_all = c[kC1], s2 = c[kC2], s3_all = c[kC3], s4 = c[kC4];
  d.row_long = c[kCLong];
  d.row_block = c[kCBlock];
  d.row_zero = c[kCZero];
  const int32_t *rid1 = sorted, *rid2 = rid1 + s1_all, *rid3 = rid2 + s2, *rid4 = rid3 + s3_all;
  const int32_t *lrid = rid4 + s4, *ridA = lrid + d.row_long, *zrid = ridA + d.row_block;
  // --- short part sizes (dasp.cu:919-955)
  int32_t common13 = s1_all < s3_all ? s1_all : s3_all;
  if (common13 / 8 >= 16)
    common13 = 8 * (common13 / 8);
  else
    common13 = 0;
  d.common_13 = common13;
  d.short_row_1 = s1_all - common13;
  d.short_row_3 = s3_all - common13;
  d.short_row_2 = s2;
  d.short_row_4 = s4;
  d.short_row_34 = d.short_row_3 + s4;
  const int32_t short_block13 = (common13 + 7) / 8;
  const int32_t short_block22 = ((s2 + 1) / 2 + 7) / 8;
  const int32_t short_block34 = (d.short_row_34 + 7) / 8;
  const int32_t tb13 = (short_block13 + 7) / 8, tb22 = (short_block22 + 7) / 8, tb34 = (short_block34 + 15) / 16;
  d.fill0_nnz_short13 = tb13 * 8 * kTile;
  d.fill0_nnz_short34 = tb34 * 16 * kTile;
  d.fill0_nnz_short22 = tb22 * 8 * kTile;
  d.fill0_nnz_short = d.short_row_1 + d.fill0_nnz_short13 + d.fill0_nnz_short34 + d.fill0_nnz_short22;
  BSP_TRY(dalloc(&d.short_val, (size_t)d.fill0_nnz_short, s));
  BSP_TRY(dalloc(&d.short_cid, (size_t)d.fill0_nnz_short, s));
  BSP_CUDA(cudaMemsetAsync(d.short_val, 0, sizeof(double) * d.fill0_nnz_short, s));
  BSP_CUDA(cudaMemsetAsync(d.short_cid, 0, sizeof(int32_t) * d.fill0_nnz_short, s));
  {
    DaspShortLayout L{d.short_row_1, s2, d.short_row_3, s4, common13, rid1, rid2, rid3, rid4,
                      d.fill0_nnz_short13, d.fill0_nnz_short34};
    const int64_t items = (int64_t)d.short_row_1 + common13 + d.short_row_3 + s4 + s2;
    if (items > 0) {
      dasp_short_fill_kernel<<<dgrid(items), 256, 0, s>>>(L, rowPtr, colIdx, values, d.short_val, d.short_cid);
      BSP_LAUNCH_CHECK();
    }
  }
  // --- long part (dasp.cu:1326-1369)
  int64_t *d_total = nullptr;
  BSP_TRY(dalloc(&d_total, 1, s));
  BSP_TRY(dalloc(&d.long_ptr_warp, (size_t)d.row_long + 1, s));
  BSP_CUDA(cudaMemsetAsync(d.long_ptr_warp, 0, sizeof(int32_t) * ((size_t)d.row_long + 1), s));
  if (d.row_long > 0) {
    dasp_long_count_kernel<<<dgrid(d.row_long), 256, 0, s>>>(d.row_long, lrid, rowPtr, d.long_ptr_warp);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(d.long_ptr_warp, d.long_ptr_warp, (int64_t)d.row_long + 1, d_total, s));
  int64_t lw = 0;
  BSP_TRY(read_i64(d_total, &lw, s));
  d.long_warps = (int32_t)lw;
  const int32_t block_num_long = (int32_t)ceil_div(lw, 4);
  d.warp_number = block_num_long * 4;
  d.fill0_nnz_long = d.warp_number * kLongChunk;
  BSP_TRY(dalloc(&d.long_val, (size_t)d.fill0_nnz_long, s));
  BSP_TRY(dalloc(&d.long_cid, (size_t)d.fill0_nnz_long, s));
  BSP_TRY(dalloc(&d.long_row_of_warp, (size_t)d.warp_number, s));
  BSP_TRY(dalloc(&d.warp_val, (size_t)d.warp_number, s));
  BSP_TRY(dalloc(&d.long_done, (size_t)d.row_long, s));
  BSP_CUDA(cudaMemsetAsync(d.long_val, 0, sizeof(double) * d.fill0_nnz_long, s));
  BSP_CUDA(cudaMemsetAsync(d.long_cid, 0, sizeof(int32_t) * d.fill0_nnz_long, s));
  BSP_CUDA(cudaMemsetAsync(d.long_row_of_warp, 0xff, sizeof(int32_t) * d.warp_number, s));
  BSP_CUDA(cudaMemsetAsync(d.long_done, 0, sizeof(int32_t) * d.row_long, s));
  if (d.row_long > 0) {
    dasp_long_fill_kernel<<<dgrid((int64_t)d.row_long * 32), 256, 0, s>>>(
        d.row_long, lrid, rowPtr, colIdx, values, d.long_ptr_warp, d.long_val, d.long_cid, d.long_row_of_warp);
    BSP_LAUNCH_CHECK();
  }
  // SpMV work split: groups of kLongGroup chunks of one row
  BSP_TRY(dalloc(&d.long_group_ptr, (size_t)d.row_long + 1, s));
  BSP_CUDA(cudaMemsetAsync(d.long_group_ptr + d.row_long, 0, sizeof(int32_t), s));
  if (d.row_long > 0) {
    dasp_long_groups_kernel<<<dgrid(d.row_long), 256, 0, s>>>(d.row_long, d.long_ptr_warp, d.long_group_ptr);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(d.long_group_ptr, d.long_group_ptr, (int64_t)d.row_long + 1, d_total, s));
  int64_t ng = 0;
  BSP_TRY(read_i64(d_total, &ng, s));
  d.long_groups = (int32_t)ng;
  BSP_TRY(dalloc(&d.long_group_info, (size_t)(ng > 0 ? 4 * ng : 4), s));
  if (d.row_long > 0) {
    dasp_group_info_kernel<<<dgrid((int64_t)d.row_long * 32), 256, 0, s>>>(
        d.row_long, d.long_group_ptr, d.long_ptr_warp, reinterpret_cast<int4 *>(d.long_group_info));
    BSP_LAUNCH_CHECK();
  }
  // --- row-block part (dasp.cu:1244, :1374-1482)
  int32_t *bkey = nullptr;
  BSP_TRY(dalloc(&bkey, (size_t)d.row_block + 1, s));
  BSP_TRY(dalloc(&d.sorted_rid, (size_t)d.row_block + 1, s));
  BSP_TRY(dalloc(&d.row_len_sorted, (size_t)d.row_block + 1, s));
  if (d.row_block > 0) {
    dasp_block_keys_kernel<<<dgrid(d.row_block), 256, 0, s>>>(d.row_block, ridA, rowPtr, block_longest, bkey,
                                                               d.sorted_rid);
    BSP_LAUNCH_CHECK();
    BSP_TRY(radix_sort_pairs(bkey, d.sorted_rid, d.row_block, bits_for(block_longest), s));
  }
  dasp_sorted_len_kernel<<<dgrid((int64_t)d.row_block + 1), 256, 0, s>>>(d.row_block, bkey, block_longest,
                                                                          d.row_len_sorted);
  BSP_LAUNCH_CHECK();
  BSP_TRY(exclusive_scan_i32(d.row_len_sorted, d.row_len_sorted, (int64_t)d.row_block + 1, nullptr, s));
  dfree(bkey, s);
  int32_t blocknum = (d.row_block + 7) / 8;
  blocknum = ((blocknum + 3) / 4) * 4;  // rowloop = 1 (dasp.cu:867, :1374-1375)
  d.blocknum = blocknum;
  BSP_TRY(dalloc(&d.block_ptr, (size_t)blocknum + 1, s));
  BSP_TRY(dalloc(&d.irreg_rpt, (size_t)d.row_block + 1, s));
  BSP_CUDA(cudaMemsetAsync(d.block_ptr, 0, sizeof(int32_t) * ((size_t)blocknum + 1), s));
  BSP_CUDA(cudaMemsetAsync(d.irreg_rpt, 0, sizeof(int32_t) * ((size_t)d.row_block + 1), s));
  if (blocknum > 0) {
    dasp_block_fill_kernel<<<dgrid(blocknum), 256, 0, s>>>(blocknum, d.row_block, d.row_len_sorted, threshold,
                                                            d.block_ptr, d.irreg_rpt);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(d.block_ptr, d.block_ptr, (int64_t)blocknum + 1, d_total, s));
  int64_t freg = 0;
  BSP_TRY(read_i64(d_total, &freg, s));
  BSP_TRY(exclusive_scan_i32(d.irreg_rpt, d.irreg_rpt, (int64_t)d.row_block + 1, d_total, s));
  int64_t nirr = 0;
  BSP_TRY(read_i64(d_total, &nirr, s));
  d.fill0_nnz_reg = (int32_t)freg;
  d.nnz_irreg = (int32_t)nirr;
  BSP_TRY(dalloc(&d.irreg_val, (size_t)d.nnz_irreg, s));
  BSP_TRY(dalloc(&d.irreg_cid, (size_t)d.nnz_irreg, s));
  BSP_TRY(dalloc(&d.reg_val, (size_t)d.fill0_nnz_reg, s));
  BSP_TRY(dalloc(&d.reg_cid, (size_t)d.fill0_nnz_reg, s));
  if (d.row_block > 0) {
    dasp_irreg_fill_kernel<<<dgrid((int64_t)d.row_block * 32), 256, 0, s>>>(
        d.row_block, d.sorted_rid, d.irreg_rpt, rowPtr, colIdx, values, d.irreg_val, d.irreg_cid);
    BSP_LAUNCH_CHECK();
  }
  if (d.fill0_nnz_reg > 0) {
    dasp_reg_fill_kernel<<<dgrid(d.fill0_nnz_reg), 256, 0, s>>>(d.fill0_nnz_reg, blocknum, d.row_block, d.block_ptr,
                                                                 d.sorted_rid, rowPtr, colIdx, values, d.reg_val,
                                                                 d.reg_cid);
    BSP_LAUNCH_CHECK();
  }
  // --- y order (dasp.cu:1289-1306)
  BSP_TRY(dalloc(&d.order_rid, (size_t)rows + 1, s));
  if (rows > 0) {
    DaspOrder O{d.row_long, d.row_block, d.short_row_1, common13, d.short_row_3, s4, s2, d.row_zero,
                lrid, d.sorted_rid, rid1, rid3, rid4, rid2, zrid};
    dasp_order_kernel<<<dgrid(rows), 256, 0, s>>>(O, d.order_rid);
    BSP_LAUNCH_CHECK();
  }
  // --- the reference's launch layout (dasp.cu:1513-1539), for drop-in parity
  const int32_t block_num_short1 = (d.short_row_1 + 127) / 128;
  d.offset_reg = block_num_long;
  d.offset_short1 = d.offset_reg + blocknum / 4;
  d.offset_short13 = d.offset_short1 + block_num_short1;
  d.offset_short34 = d.offset_short13 + tb13;
  d.offset_short22 = d.offset_short34 + tb34;
  d.block_num_all = d.offset_short22 + tb22;
  d.short_block13 = short_block13;
  d.short_block34 = short_block34;
  d.short_block22 = short_block22;
  dfree(key, s);
  dfree(cnt, s);
  dfree(d_total, s);
  dfree(sorted, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  *out = d;
  return BSP_OK;
}

// ---------------------------------------------------------------------------
// Fused SpMV.  Grid sections (CTAs of 256 threads = 8 warps), in order:
// long-row groups (warp each, up to 4 chunks of 64), row blocks (warp each),
// len-1 rows (8 per thread), 1&3 tile slots (2 per thread), 3/4 tile rows
// (2 per thread), 2&2 tile rows (2 per thread), empty rows (thread each).
// Every thread issues all of its loads before the dependent x gathers, so
// each warp keeps several independent memory requests in flight.
struct DaspSections {
  int32_t long_cta, reg_cta, s1_cta, t13_cta, t34_cta, t22_cta, zero_cta;
};
constexpr int kS1PerThread = 4;
constexpr int kShortPerThread = 2;

// Device-scope atomic add with acquire-release ordering: the caller's earlier
// stores are visible to whoever acquires through this counter later, and the
// caller sees every store released into it before.
__device__ __forceinline__ int32_t atomic_add_acq_rel(int32_t *p, int32_t v) {
  int32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// y slot k -> element index (order_rid when the output is not permuted)
__device__ __forceinline__ int32_t dasp_yidx(const int32_t *outIdx, int64_t k) {
  return outIdx ? __ldg(outIdx + k) : (int32_t)k;
}

__device__ __forceinline__ void dasp_put(double *y, int32_t yi, double v, double alpha, double beta) {
  double r = alpha * v;
  if (beta != 0.0) r += beta * y[yi];
  y[yi] = r;
}

template <bool ALIGNED>
__device__ __forceinline__ f64x4 dasp_ld4(const double *p) {
  if (ALIGNED) return ld_stream_f64x4(p);
  return f64x4{__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)};
}

// 32 registers (8 CTAs of 256 per SM): every section waits on dependent
// gathers, so resident warps matter more than per-thread batching; at 64
// registers (4 CTAs) the kernel kept half the warps and took 82-84 us on the
// 2M-row power-law matrix.
template <bool SHORT_ALIGNED>
__global__ void __launch_bounds__(256, 6) dasp_spmv_kernel(bsp_dasp D, DaspSections S, const double *__restrict__ x,
                                                        double *__restrict__ y, const int32_t *__restrict__ outIdx,
                                                        double alpha, double beta) {
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  int32_t b = blockIdx.x;
  if (b < S.long_cta) {
    const int64_t g = (int64_t)b * 8 + wib;
    if (g >= D.long_groups) return;
    const int4 gi = __ldg(reinterpret_cast<const int4 *>(D.long_group_info) + g);
    const int32_t row = gi.x, c0 = gi.y, g0 = gi.z, nc = gi.w & 15, ng = gi.w >> 4;
    const uint64_t pol = evict_first_policy();
    const int32_t yi = lane == 0 ? dasp_yidx(outIdx, row) : 0;
    double2 v[kLongGroup];
    int2 c[kLongGroup];
#pragma unroll
    for (int k = 0; k < kLongGroup; ++k)
      if (k < nc) {
        v[k] = ld_stream_f64x2(D.long_val + (int64_t)(c0 + k) * kLongChunk + 2 * lane, pol);
        c[k] = __ldg(reinterpret_cast<const int2 *>(D.long_cid + (int64_t)(c0 + k) * kLongChunk) + lane);
      }
    double p = 0.0;
#pragma unroll
    for (int k = 0; k < kLongGroup; ++k)
      if (k < nc) p = fma(v[k].y, ld_x(x + c[k].y), fma(v[k].x, ld_x(x + c[k].x), p));
    p = warp_sum(p);
    if (ng == 1) {  // the whole row in this warp
      if (lane == 0) dasp_put(y, yi, p, alpha, beta);
      return;
    }
    // publish the partial with a release increment; the warp that brings the
    // counter to ng acquires every other group's partial and sums them
    int32_t last = 0;
    if (lane == 0) {
      D.warp_val[g] = p;
      last = atomic_add_acq_rel(&D.long_done[row], 1) == ng - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {  // every group of this row is stored: sum them in order
      __syncwarp();
      double sum = 0.0;
      for (int32_t k = g0 + lane; k < g0 + ng; k += 32) sum += __ldcg(D.warp_val + k);
      sum = warp_sum(sum);
      if (lane == 0) {
        dasp_put(y, yi, sum, alpha, beta);
        D.long_done[row] = 0;  // ready for the next call
      }
    }
    return;
  }
  b -= S.long_cta;
  if (b < S.reg_cta) {
    const int64_t bid = (int64_t)b * 8 + wib;
    if (bid * 8 >= D.row_block) return;
    // lane: tile slot t (4 tiles per step, two steps in flight), row r; the
    // row's irregular tail is split over the same 4 slots
    const int t = lane >> 3, r = lane & 7;
    const int64_t row = bid * 8 + r;
    const bool live = row < D.row_block;
    const int32_t p0 = D.block_ptr[bid], p1 = D.block_ptr[bid + 1];
    const int32_t i0 = live ? __ldg(D.irreg_rpt + row) : 0, i1 = live ? __ldg(D.irreg_rpt + row + 1) : 0;
    const int32_t yi = (live && t == 0) ? dasp_yidx(outIdx, D.row_long + row) : 0;
    double acc = 0.0;
    int32_t o = p0 + t * kTile;
    int32_t j = i0 + t;
    for (; o + 4 * kTile < p1; o += 8 * kTile) {
      const f64x4 v0 = ld_stream_f64x4(D.reg_val + o + r * 4);
      const int4 c0 = __ldg(reinterpret_cast<const int4 *>(D.reg_cid + o + r * 4));
      const f64x4 v1 = ld_stream_f64x4(D.reg_val + o + 4 * kTile + r * 4);
      const int4 c1 = __ldg(reinterpret_cast<const int4 *>(D.reg_cid + o + 4 * kTile + r * 4));
      acc = fma(v0.x, ld_x(x + c0.x), acc);
      acc = fma(v0.y, ld_x(x + c0.y), acc);
      acc = fma(v0.z, ld_x(x + c0.z), acc);
      acc = fma(v0.w, ld_x(x + c0.w), acc);
      acc = fma(v1.x, ld_x(x + c1.x), acc);
      acc = fma(v1.y, ld_x(x + c1.y), acc);
      acc = fma(v1.z, ld_x(x + c1.z), acc);
      acc = fma(v1.w, ld_x(x + c1.w), acc);
    }
    {  // last step of tiles together with the first irregular element
      const bool has_t = o < p1, has_i = j < i1;
      f64x4 v = {0.0, 0.0, 0.0, 0.0};
      int4 c = {0, 0, 0, 0};
      double iv = 0.0;
      int32_t ic = 0;
      if (has_t) {
        v = ld_stream_f64x4(D.reg_val + o + r * 4);
        c = __ldg(reinterpret_cast<const int4 *>(D.reg_cid + o + r * 4));
      }
      if (has_i) {
        iv = __ldg(D.irreg_val + j);
        ic = __ldg(D.irreg_cid + j);
      }
      if (has_t) {
        acc = fma(v.x, ld_x(x + c.x), acc);
        acc = fma(v.y, ld_x(x + c.y), acc);
        acc = fma(v.z, ld_x(x + c.z), acc);
        acc = fma(v.w, ld_x(x + c.w), acc);
      }
      if (has_i) acc = fma(iv, ld_x(x + ic), acc);
    }
    for (j += 4; j < i1; j += 4) acc = fma(__ldg(D.irreg_val + j), ld_x(x + __ldg(D.irreg_cid + j)), acc);
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (t == 0 && live) dasp_put(y, yi, acc, alpha, beta);
    return;
  }
  b -= S.reg_cta;
  const int64_t ybase = (int64_t)D.row_long + D.row_block;
  if (b < S.s1_cta) {
    const int64_t i0 = (int64_t)b * 256 * kS1PerThread + threadIdx.x;
    double v[kS1PerThread];
    int32_t c[kS1PerThread];
    int32_t yi[kS1PerThread];
    const uint64_t pol = evict_first_policy();
#pragma unroll
    for (int k = 0; k < kS1PerThread; ++k) {
      const int64_t i = i0 + k * 256;
      if (i < D.short_row_1) {
        v[k] = ld_stream_f64(D.short_val + i, pol);
        c[k] = ld_stream_s32(D.short_cid + i, pol);
        yi[k] = dasp_yidx(outIdx, ybase + i);
      }
    }
#pragma unroll
    for (int k = 0; k < kS1PerThread; ++k) {
      const int64_t i = i0 + k * 256;
      if (i < D.short_row_1) dasp_put(y, yi[k], v[k] * ld_x(x + c[k]), alpha, beta);
    }
    return;
  }
  b -= S.s1_cta;
  const double *sv = D.short_val + D.short_row_1;
  const int32_t *sc = D.short_cid + D.short_row_1;
  if (b < S.t13_cta) {
    // slot s: tile s/16, q = s%16: q < 8 the len-1 row of tile row q, else
    // the len-3 row of tile row q-8
    const int64_t s0 = (int64_t)b * 256 * kShortPerThread + threadIdx.x;
    const int64_t ns = 2 * (int64_t)D.common_13;
    double v[kShortPerThread][3];
    int32_t c[kShortPerThread][3];
    int32_t yi[kShortPerThread];
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < ns) {
        yi[k] = dasp_yidx(outIdx, ybase + D.short_row_1 + s);
        const int q = (int)(s & 15), j = q & 7;
        const int64_t o = (s >> 4) * kTile + j * 4;
        if (q < 8) {
          v[k][0] = __ldg(sv + o);
          c[k][0] = __ldg(sc + o);
        } else {
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            v[k][m] = __ldg(sv + o + 1 + m);
            c[k][m] = __ldg(sc + o + 1 + m);
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < ns) {
        double a;
        if ((s & 15) < 8)
          a = v[k][0] * ld_x(x + c[k][0]);
        else
          a = fma(v[k][2], ld_x(x + c[k][2]), fma(v[k][1], ld_x(x + c[k][1]), v[k][0] * ld_x(x + c[k][0])));
        dasp_put(y, yi[k], a, alpha, beta);
      }
    }
    return;
  }
  b -= S.t13_cta;
  const double *sv34 = sv + D.fill0_nnz_short13;
  const int32_t *sc34 = sc + D.fill0_nnz_short13;
  if (b < S.t34_cta) {
    // slot s = row s%8 of tile s/8: 4 values at sv34 + 4s
    const int64_t s0 = (int64_t)b * 256 * kShortPerThread + threadIdx.x;
    f64x4 v[kShortPerThread];
    int4 c[kShortPerThread];
    int32_t yi[kShortPerThread];
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < D.short_row_34) {
        yi[k] = dasp_yidx(outIdx, ybase + D.short_row_1 + 2 * (int64_t)D.common_13 + s);
        v[k] = dasp_ld4<SHORT_ALIGNED>(sv34 + s * 4);
        c[k] = make_int4(__ldg(sc34 + s * 4), __ldg(sc34 + s * 4 + 1), __ldg(sc34 + s * 4 + 2),
                         __ldg(sc34 + s * 4 + 3));
      }
    }
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < D.short_row_34) {
        double a = v[k].x * ld_x(x + c[k].x);
        a = fma(v[k].y, ld_x(x + c[k].y), a);
        a = fma(v[k].z, ld_x(x + c[k].z), a);
        a = fma(v[k].w, ld_x(x + c[k].w), a);
        dasp_put(y, yi[k], a, alpha, beta);
      }
    }
    return;
  }
  b -= S.t34_cta;
  const double *sv22 = sv34 + D.fill0_nnz_short34;
  const int32_t *sc22 = sc34 + D.fill0_nnz_short34;
  if (b < S.t22_cta) {
    // slot s: tile s/16, q = s%16 -> positions (q%8)*4 + (q/8)*2 + {0,1}
    const int64_t s0 = (int64_t)b * 256 * kShortPerThread + threadIdx.x;
    double2 v[kShortPerThread];
    int2 c[kShortPerThread];
    int32_t yi[kShortPerThread];
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < D.short_row_2) {
        yi[k] = dasp_yidx(outIdx, ybase + D.short_row_1 + 2 * (int64_t)D.common_13 + D.short_row_34 + s);
        const int q = (int)(s & 15);
        const int64_t o = (s >> 4) * kTile + (q & 7) * 4 + (q >> 3) * 2;
        v[k] = make_double2(__ldg(sv22 + o), __ldg(sv22 + o + 1));
        c[k] = make_int2(__ldg(sc22 + o), __ldg(sc22 + o + 1));
      }
    }
#pragma unroll
    for (int k = 0; k < kShortPerThread; ++k) {
      const int64_t s = s0 + k * 256;
      if (s < D.short_row_2) {
        const double a = fma(v[k].y, ld_x(x + c[k].y), v[k].x * ld_x(x + c[k].x));
        dasp_put(y, yi[k], a, alpha, beta);
      }
    }
    return;
  }
  b -= S.t22_cta;
  {
    const int64_t i = (int64_t)b * 256 + threadIdx.x;
    if (i < D.row_zero) dasp_put(y, dasp_yidx(outIdx, (int64_t)D.rows - D.row_zero + i), 0.0, alpha, beta);
  }
}

bsp_status dasp_spmv_impl(const bsp_dasp *d, const double *x, double *y, double alpha, double beta,
                          int32_t permuted_output, cudaStream_t s) {
  if (d->rows == 0) return BSP_OK;
  DaspSections S;
  S.long_cta = (int32_t)ceil_div(d->long_groups, 8);
  S.reg_cta = (int32_t)ceil_div(ceil_div(d->row_block, 8), 8);
  S.s1_cta = (int32_t)ceil_div(d->short_row_1, 256 * kS1PerThread);
  S.t13_cta = (int32_t)ceil_div(2 * (int64_t)d->common_13, 256 * kShortPerThread);
  S.t34_cta = (int32_t)ceil_div(d->short_row_34, 256 * kShortPerThread);
  S.t22_cta = (int32_t)ceil_div(d->short_row_2, 256 * kShortPerThread);
  S.zero_cta = (int32_t)ceil_div(d->row_zero, 256);
  const int64_t grid = (int64_t)S.long_cta + S.reg_cta + S.s1_cta + S.t13_cta + S.t34_cta + S.t22_cta + S.zero_cta;
  if (grid == 0) return BSP_OK;
  const int32_t *outIdx = permuted_output ? nullptr : d->order_rid;
  const bool aligned = ((uintptr_t)(d->short_val + d->short_row_1 + d->fill0_nnz_short13) & 31) == 0;
  if (aligned)
    dasp_spmv_kernel<true><<<(unsigned)grid, 256, 0, s>>>(*d, S, x, y, outIdx, alpha, beta);
  else
    dasp_spmv_kernel<false><<<(unsigned)grid, 256, 0, s>>>(*d, S, x, y, outIdx, alpha, beta);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_csr2dasp(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                   const int32_t *colIdx, const double *values, double threshold,
                                   int32_t block_longest, bsp_dasp *out, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out, "null output descriptor");
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  BSP_CHECK_ARG(rowPtr && (nnz == 0 || (colIdx && values)), "null pointer");
  // threshold <= 0 would keep an empty tile forever (dasp.cu:1395-1411 loops
  // while block_nnz >= threshold*32, and a padding block has block_nnz 0).
  BSP_CHECK_ARG(threshold > 0.0, "threshold must be > 0");
  BSP_CHECK_ARG(block_longest >= 1, "block_longest must be >= 1");
  return csr2dasp_impl(rows, cols, nnz, rowPtr, colIdx, values, threshold, block_longest, out, as_stream(stream));
}

extern "C" bsp_status bsp_dasp_free(bsp_dasp *d) {
  clear_error();
  if (!d) return BSP_OK;
  cudaStream_t s = 0;
  dfree(d->long_val, s);
  dfree(d->long_cid, s);
  dfree(d->long_ptr_warp, s);
  dfree(d->long_row_of_warp, s);
  dfree(d->warp_val, s);
  dfree(d->long_done, s);
  dfree(d->reg_val, s);
  dfree(d->reg_cid, s);
  dfree(d->block_ptr, s);
  dfree(d->irreg_val, s);
  dfree(d->irreg_cid, s);
  dfree(d->irreg_rpt, s);
  dfree(d->short_val, s);
  dfree(d->short_cid, s);
  dfree(d->order_rid, s);
  dfree(d->sorted_rid, s);
  dfree(d->row_len_sorted, s);
  dfree(d->long_group_ptr, s);
  dfree(d->long_group_info, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_dasp_spmv(const bsp_dasp *d, const double *x, double *y, double alpha, double beta,
                                    int32_t permuted_output, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(d && x && y, "null pointer");
  return dasp_spmv_impl(d, x, y, alpha, beta, permuted_output, as_stream(stream));
}
