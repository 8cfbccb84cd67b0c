// cuSPARSE SpMV baselines under the reference's names (include/cusp.h:3-6,
// src/cusparse.cu:35-390), for comparison runs only: the library's own paths
// never call cuSPARSE.  Device memory goes through libbspmv's C ABI.
#include <cusparse.h>
#include <stdio.h>

#include <chrono>
#include <vector>

#include "benchsp_compat.hpp"
#include "bsp.h"

namespace {

bool sp_ok(cusparseStatus_t s, const char *what) {
  if (s == CUSPARSE_STATUS_SUCCESS) return true;
  fprintf(stderr, "%s: %s\n", what, cusparseGetErrorString(s));
  return false;
}

bool b_ok(bsp_status s, const char *what) {
  if (s == BSP_OK) return true;
  fprintf(stderr, "%s: %s\n", what, bsp_last_error());
  return false;
}

struct Buf {
  void *p = nullptr;
  Buf() = default;
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
  ~Buf() {
    if (p) bsp_device_free(p);
  }
  bool alloc(size_t b) { return b_ok(bsp_device_alloc(&p, b ? b : 16), "bsp_device_alloc"); }
  template <typename T>
  bool up(const T *h, size_t n) {
    return alloc(n * sizeof(T)) && (n == 0 || b_ok(bsp_memcpy_h2d(p, h, n * sizeof(T)), "bsp_memcpy_h2d"));
  }
  template <typename T>
  bool down(T *h, size_t n) {
    return n == 0 || b_ok(bsp_memcpy_d2h(h, p, n * sizeof(T)), "bsp_memcpy_d2h");
  }
};

// y = A*x with cuSPARSE's generic SpMV.  idx: index type of both arrays;
// vt: value type of A/x/y; ct: compute type (alpha/beta have this type).
bool generic_spmv(int64_t rows, int64_t cols, int64_t nnz, void *rp, void *ci, void *va, void *x, void *y,
                  cusparseIndexType_t idx, cudaDataType vt, cudaDataType ct, const void *alpha, const void *beta,
                  int warm, int repeat, double *avg_us) {
  cusparseHandle_t h = nullptr;
  cusparseSpMatDescr_t A = nullptr;
  cusparseDnVecDescr_t vx = nullptr, vy = nullptr;
  bool good = sp_ok(cusparseCreate(&h), "cusparseCreate") &&
              sp_ok(cusparseCreateCsr(&A, rows, cols, nnz, rp, ci, va, idx, idx, CUSPARSE_INDEX_BASE_ZERO, vt),
                    "cusparseCreateCsr") &&
              sp_ok(cusparseCreateDnVec(&vx, cols, x, vt), "cusparseCreateDnVec") &&
              sp_ok(cusparseCreateDnVec(&vy, rows, y, vt), "cusparseCreateDnVec");
  size_t wsb = 0;
  Buf ws;
  if (good)
    good = sp_ok(cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, vx, beta, vy, ct,
                                         CUSPARSE_SPMV_ALG_DEFAULT, &wsb),
                 "cusparseSpMV_bufferSize") &&
           ws.alloc(wsb);
  auto run = [&] {
    return sp_ok(cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, vx, beta, vy, ct,
                              CUSPARSE_SPMV_ALG_DEFAULT, ws.p),
                 "cusparseSpMV") &&
           b_ok(bsp_device_sync(), "bsp_device_sync");
  };
  for (int i = 0; good && i < warm; ++i) good = run();
  if (good) {
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; good && i < repeat; ++i) good = run();
    const auto t1 = std::chrono::steady_clock::now();
    if (avg_us) *avg_us = repeat > 0 ? std::chrono::duration<double, std::micro>(t1 - t0).count() / repeat : 0.0;
    if (repeat <= 0) good = run();
  }
  if (vy) cusparseDestroyDnVec(vy);
  if (vx) cusparseDestroyDnVec(vx);
  if (A) cusparseDestroySpMat(A);
  if (h) cusparseDestroy(h);
  return good;
}

}  // namespace

int cusparse_spmv(int *A_csrOffsets, int64_t *A_columns, float *A_values, float *x, float *y, int64_t row,
                  int64_t col, int64_t nnz) {
  std::vector<int32_t> ci(nnz);
  for (int64_t i = 0; i < nnz; ++i) ci[i] = (int32_t)A_columns[i];
  Buf rp, cd, va, xd, yd;
  const float a = 1.0f, b = 0.0f;
  if (!rp.up(A_csrOffsets, (size_t)row + 1) || !cd.up(ci.data(), ci.size()) || !va.up(A_values, nnz) ||
      !xd.up(x, col) || !yd.alloc(sizeof(float) * row) ||
      !generic_spmv(row, col, nnz, rp.p, cd.p, va.p, xd.p, yd.p, CUSPARSE_INDEX_32I, CUDA_R_32F, CUDA_R_32F, &a, &b,
                    0, 0, nullptr) ||
      !yd.down(y, row))
    return 1;
  return 0;
}

int cusparse_spmv_fp64(int64_t *hA_csrOffsets, int64_t *hA_columns, double *hA_values, double *hX, double *hY,
                       int64_t A_num_rows, int64_t A_num_cols, int64_t A_nnz, int repeat, double &avg_time) {
  Buf rp, ci, va, xd, yd;
  const double a = 1.0, b = 0.0;
  if (!rp.up(hA_csrOffsets, (size_t)A_num_rows + 1) || !ci.up(hA_columns, A_nnz) || !va.up(hA_values, A_nnz) ||
      !xd.up(hX, A_num_cols) || !yd.alloc(sizeof(double) * A_num_rows) ||
      !generic_spmv(A_num_rows, A_num_cols, A_nnz, rp.p, ci.p, va.p, xd.p, yd.p, CUSPARSE_INDEX_64I, CUDA_R_64F,
                    CUDA_R_64F, &a, &b, 10, repeat, &avg_time) ||
      !yd.down(hY, A_num_rows))
    return 1;
  return 0;
}

int cusparse_spmv_fp16(int *hA_csrOffsets, int32_t *hA_columns, half *hA_values, half *hX, half *hY,
                       int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz) {
  Buf rp, ci, va, xd, yd;
  const float a = 1.0f, b = 0.0f;
  if (!rp.up(hA_csrOffsets, (size_t)A_num_rows + 1) || !ci.up(hA_columns, A_nnz) || !va.up(hA_values, A_nnz) ||
      !xd.up(hX, A_num_cols) || !yd.alloc(sizeof(half) * A_num_rows) ||
      !generic_spmv(A_num_rows, A_num_cols, A_nnz, rp.p, ci.p, va.p, xd.p, yd.p, CUSPARSE_INDEX_32I, CUDA_R_16F,
                    CUDA_R_32F, &a, &b, 0, 0, nullptr) ||
      !yd.down(hY, A_num_rows))
    return 1;
  return 0;
}

void cusparse_spmv_fp16_warpper(int *hA_csrOffsets, int32_t *hA_columns, float *hA_values32, float *hX32,
                                float *hY32, int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz) {
  std::vector<half> v(A_nnz), x(A_num_cols), y(A_num_rows);
  for (int32_t i = 0; i < A_nnz; ++i) v[i] = __float2half(hA_values32[i]);
  for (int32_t i = 0; i < A_num_cols; ++i) x[i] = __float2half(hX32[i]);
  if (cusparse_spmv_fp16(hA_csrOffsets, hA_columns, v.data(), x.data(), y.data(), A_num_rows, A_num_cols, A_nnz) ==
      0)
    for (int32_t i = 0; i < A_num_rows; ++i) hY32[i] = __half2float(y[i]);
}
