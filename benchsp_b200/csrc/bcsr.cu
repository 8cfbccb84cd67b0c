// Fixed-tile BCSR (BCSRFormat, reference include/matrixFormat.hpp:16-30,
// built by csrToBcsr, utils/utils.hpp:10-123): conversion on the device and a
// generic tile SpMV.
//
// csrToBcsr walks a dense rowRegions x colRegions occupancy table on the
// host (O(rowRegions*colRegions) memory and time; 4.3e9 entries for the
// n = 2^20 matrices of the SpMM benchmark).  The device conversion here
// builds the same arrays -- block columns ascending per block-row, tm x tk
// row-major values, block ordinals in row-major order -- from the
// sort-free canonical-element construction of bsr.cu, in O(nnz log).  The
// dense relativeBlockIndexMapping is produced only on request.
//
// SpMV replaces bcsr_spmv_kernel / bcsr_spmv_kernel_column_by_column
// (reference src/bcsr.cu:22, :161, fixed 2x2 / 3x3 tiles) with one kernel for
// any tile shape: one thread per (block-row, row in tile), its tk values of
// each block contiguous.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

bsp_status csr2blocks(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx, const double *values,
                      int32_t tm, int32_t tk, int32_t *blc_num_out, int32_t **blcPtr, int32_t **blcIdx,
                      double **blcVal, uint16_t **map16, uint64_t **map64, cudaStream_t s);

__global__ void bcsr_mapping_kernel(int32_t nr, int32_t nc, const int32_t *__restrict__ rp,
                                    const int32_t *__restrict__ ci, int32_t *__restrict__ mapping) {
  for (int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; br < nr; br += (int64_t)gridDim.x * blockDim.x)
    for (int32_t k = rp[br]; k < rp[br + 1]; ++k) mapping[br * (int64_t)nc + ci[k]] = k;
}

__global__ void bcsr_spmv_kernel(int32_t row, int32_t col, int32_t nr, int32_t tm, int32_t tk,
                                 const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                 const double *__restrict__ val, const double *__restrict__ x,
                                 double *__restrict__ y, double alpha, double beta) {
  const int64_t total = (int64_t)nr * tm;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t br = t / tm;
    const int r = (int)(t % tm);
    const int64_t yi = br * tm + r;
    if (yi >= row) continue;
    double acc = 0.0;
    for (int32_t k = rp[br]; k < rp[br + 1]; ++k) {
      const double *v = val + (int64_t)k * tm * tk + (int64_t)r * tk;
      const int64_t c0 = (int64_t)ci[k] * tk;
      for (int c = 0; c < tk; ++c)
        if (c0 + c < col) acc = fma(v[c], __ldg(&x[c0 + c]), acc);
    }
    double res = alpha * acc;
    if (beta != 0.0) res += beta * y[yi];
    y[yi] = res;
  }
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_csr2bcsr(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                   const int32_t *colIdx, const double *values, int32_t tile_m, int32_t tile_k,
                                   int32_t with_mapping, bsp_bcsr *out, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out, "null output descriptor");
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  BSP_CHECK_ARG(tile_m >= 1 && tile_k >= 1 && tile_m <= 64 && tile_k <= 64, "tile sizes must be in [1, 64]");
  BSP_CHECK_ARG(rowPtr && (nnz == 0 || (colIdx && values)), "null pointer");
  cudaStream_t s = as_stream(stream);
  bsp_bcsr b{};
  b.row = rows;
  b.col = cols;
  b.nnz = nnz;
  b.TILE_M = tile_m;
  b.TILE_K = tile_k;
  b.TILE_N = tile_k;
  b.rowRegions = (int32_t)ceil_div(rows, tile_m);
  b.colRegions = (int32_t)ceil_div(cols, tile_k);
  b.block_row = b.rowRegions;
  b.block_col = b.colRegions;
  b.blockNum = (int64_t)b.rowRegions * b.colRegions;
  if (with_mapping && b.blockNum > ((int64_t)1 << 31))
    BSP_FAIL(BSP_ERR_UNSUPPORTED, "dense block mapping larger than 2^31 entries");
  BSP_TRY(csr2blocks(rows, nnz, rowPtr, colIdx, values, tile_m, tile_k, &b.nonzeroBlocks, &b.bcsrRowPtr,
                     &b.bcsrcolIdx, &b.values, nullptr, nullptr, s));
  b.elemCount = b.nonzeroBlocks * tile_m * tile_k;
  if (with_mapping) {
    BSP_TRY(dalloc(&b.relativeBlockIndexMapping, (size_t)b.blockNum, s));
    BSP_CUDA(cudaMemsetAsync(b.relativeBlockIndexMapping, 0xff, sizeof(int32_t) * (size_t)b.blockNum, s));
    if (b.rowRegions > 0) {
      int64_t g = ceil_div(b.rowRegions, 256);
      if (g > 4096) g = 4096;
      bcsr_mapping_kernel<<<(unsigned)g, 256, 0, s>>>(b.rowRegions, b.colRegions, b.bcsrRowPtr, b.bcsrcolIdx,
                                                     b.relativeBlockIndexMapping);
      BSP_LAUNCH_CHECK();
    }
  }
  BSP_CUDA(cudaStreamSynchronize(s));
  *out = b;
  return BSP_OK;
}

extern "C" bsp_status bsp_bcsr_free(bsp_bcsr *b) {
  clear_error();
  if (!b) return BSP_OK;
  cudaStream_t s = 0;
  dfree(b->bcsrRowPtr, s);
  dfree(b->bcsrcolIdx, s);
  dfree(b->relativeBlockIndexMapping, s);
  dfree(b->values, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_bcsr_spmv(const bsp_bcsr *b, const double *x, double *y, double alpha, double beta,
                                    bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(b && x && y, "null pointer");
  if (b->rowRegions == 0) return BSP_OK;
  const int64_t total = (int64_t)b->rowRegions * b->TILE_M;
  int64_t g = ceil_div(total, 256);
  if (g > (int64_t)sm_count() * 32) g = (int64_t)sm_count() * 32;
  bcsr_spmv_kernel<<<(unsigned)g, 256, 0, as_stream(stream)>>>(b->row, b->col, b->rowRegions, b->TILE_M, b->TILE_K,
                                                              b->bcsrRowPtr, b->bcsrcolIdx, b->values, x, y, alpha,
                                                              beta);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}
