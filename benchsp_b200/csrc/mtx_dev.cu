// Triplets -> CSR on the device for bsp_mtx_csr (mtx.cpp parses the file).
//
// Order: rows ascending, columns ascending within a row, triplet order among
// equal (row, col).  Two stable LSD radix sorts of the triplet index give it:
// first by column, then by row (a stable sort by the major key after one by
// the minor key).  Triplets already in (col, row) order skip the first sort;
// triplets already in (row, col) order are copied as they are.  The row
// pointer is a lower bound of each row in the sorted row keys, one thread
// per row.
#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

__global__ void mtx_iota_kernel(int32_t *__restrict__ a, int64_t n) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    a[k] = (int32_t)k;
}

__global__ void mtx_gather_key_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ idx,
                                      int32_t *__restrict__ out, int64_t n) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    out[k] = src[idx[k]];
}

__global__ void mtx_gather_kernel(const int32_t *__restrict__ col, const double *__restrict__ val,
                                  const int32_t *__restrict__ idx, int32_t *__restrict__ colIdx,
                                  double *__restrict__ values, int64_t n) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = idx[k];
    colIdx[k] = col[i];
    values[k] = val[i];
  }
}

// rowPtr[r] = number of sorted keys below r, for r in [0, rows].
__global__ void mtx_rowptr_kernel(const int32_t *__restrict__ rk, int64_t n, int32_t rows,
                                  int32_t *__restrict__ rowPtr) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= rows; r += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (rk[mid] < r)
        lo = mid + 1;
      else
        hi = mid;
    }
    rowPtr[r] = (int32_t)lo;
  }
}

static unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), 148 * 16)); }

bsp_status mtx_csr_device(int32_t rows, int32_t cols, int64_t nnz, const int32_t *r, const int32_t *c,
                          const double *v, bool sorted, bool col_sorted, int32_t *rowPtr, int32_t *colIdx,
                          double *values, cudaStream_t s) {
  if (nnz == 0) {
    BSP_CUDA(cudaMemsetAsync(rowPtr, 0, sizeof(int32_t) * ((size_t)rows + 1), s));
    BSP_CUDA(cudaStreamSynchronize(s));
    return BSP_OK;
  }
  int32_t *dr = nullptr, *dc = nullptr, *idx = nullptr, *key = nullptr;
  double *dv = nullptr;
  bsp_status st = BSP_OK;
  auto done = [&](bsp_status x) {
    dfree(dr, s);
    dfree(dc, s);
    dfree(idx, s);
    dfree(key, s);
    dfree(dv, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (x == BSP_OK && e != cudaSuccess) {
      set_error(std::string("mtx_csr_device: ") + cudaGetErrorString(e));
      return BSP_ERR_CUDA;
    }
    return x;
  };
#define MTX_TRY(call)             \
  do {                            \
    st = (call);                  \
    if (st != BSP_OK) return done(st); \
  } while (0)
#define MTX_CUDA(call)                                                          \
  do {                                                                          \
    const cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                                    \
      set_error(std::string("mtx_csr_device: " #call " -> ") + cudaGetErrorString(e_)); \
      return done(BSP_ERR_CUDA);                                                \
    }                                                                           \
  } while (0)
  MTX_TRY(dalloc(&dr, (size_t)nnz, s));
  MTX_CUDA(cudaMemcpyAsync(dr, r, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
  const unsigned g = grid_for(nnz);
  if (sorted) {
    MTX_CUDA(cudaMemcpyAsync(colIdx, c, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
    MTX_CUDA(cudaMemcpyAsync(values, v, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    mtx_rowptr_kernel<<<grid_for((int64_t)rows + 1), 256, 0, s>>>(dr, nnz, rows, rowPtr);
    MTX_CUDA(cudaGetLastError());
    return done(BSP_OK);
  }
  MTX_TRY(dalloc(&dc, (size_t)nnz, s));
  MTX_TRY(dalloc(&idx, (size_t)nnz, s));
  MTX_TRY(dalloc(&key, (size_t)nnz, s));
  MTX_TRY(dalloc(&dv, (size_t)nnz, s));
  MTX_CUDA(cudaMemcpyAsync(dc, c, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
  MTX_CUDA(cudaMemcpyAsync(dv, v, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
  mtx_iota_kernel<<<g, 256, 0, s>>>(idx, nnz);
  MTX_CUDA(cudaGetLastError());
  if (!col_sorted) {
    MTX_CUDA(cudaMemcpyAsync(key, dc, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s));
    MTX_TRY(radix_sort_pairs(key, idx, nnz, bits_for(std::max(0, cols - 1)), s));
  }
  mtx_gather_key_kernel<<<g, 256, 0, s>>>(dr, idx, key, nnz);
  MTX_CUDA(cudaGetLastError());
  MTX_TRY(radix_sort_pairs(key, idx, nnz, bits_for(std::max(0, rows - 1)), s));
  mtx_gather_kernel<<<g, 256, 0, s>>>(dc, dv, idx, colIdx, values, nnz);
  MTX_CUDA(cudaGetLastError());
  mtx_rowptr_kernel<<<grid_for((int64_t)rows + 1), 256, 0, s>>>(key, nnz, rows, rowPtr);
  MTX_CUDA(cudaGetLastError());
#undef MTX_TRY
#undef MTX_CUDA
  return done(BSP_OK);
}

}  // namespace bsp
