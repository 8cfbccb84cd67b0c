// The reference's host-pointer operator functions (include/csrspmv.h,
// spmv.h, amgT.h, bcsr.h, dasp.h, smat.h) over the C ABI of libbspmv.  Each
// call uploads its inputs, converts on the device where the reference
// converts, runs the timed launches, downloads the result and frees what it
// allocated.  Semantics and deliberate differences: benchsp_compat.hpp.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "benchsp_compat.hpp"
#include "bsp.h"

namespace {

bool g_accumulate = false;

bool ok(bsp_status s, const char *what) {
  if (s == BSP_OK) return true;
  fprintf(stderr, "%s: %s\n", what, bsp_last_error());
  return false;
}

// Owned device buffer.
struct Dev {
  void *p = nullptr;
  Dev() = default;
  Dev(const Dev &) = delete;
  Dev &operator=(const Dev &) = delete;
  ~Dev() {
    if (p) bsp_device_free(p);
  }
  bool alloc(size_t bytes) { return ok(bsp_device_alloc(&p, bytes ? bytes : 16), "bsp_device_alloc"); }
  template <typename T>
  bool upload(const T *h, size_t n) {
    if (!alloc(n * sizeof(T))) return false;
    return n == 0 || ok(bsp_memcpy_h2d(p, h, n * sizeof(T)), "bsp_memcpy_h2d");
  }
  template <typename T>
  bool download(T *h, size_t n) const {
    return n == 0 || ok(bsp_memcpy_d2h(h, p, n * sizeof(T)), "bsp_memcpy_d2h");
  }
  template <typename T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// Runs `warm` untimed and `repeat` timed launches, each followed by a device
// synchronize (the reference's timing loop); returns microseconds per launch,
// or -1 on failure.
template <typename F>
double timed(int warm, int repeat, F &&launch) {
  for (int i = 0; i < warm; ++i)
    if (!launch() || !ok(bsp_device_sync(), "bsp_device_sync")) return -1.0;
  if (repeat <= 0) return 0.0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < repeat; ++i)
    if (!launch() || !ok(bsp_device_sync(), "bsp_device_sync")) return -1.0;
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double, std::micro>(t1 - t0).count() / repeat;
}

// Timed launches into a scratch y, then the result launch into y_dev (which
// holds the caller's y when accumulating).
template <typename F>
bool run_result(int warm, int repeat, Dev &y_dev, size_t ybytes, double &avg_time, F &&launch_into,
                bool acc = g_accumulate) {
  Dev scratch;
  if (!scratch.alloc(ybytes)) return false;
  const double t = timed(warm, repeat, [&] { return launch_into(scratch.p, 0.0); });
  if (t < 0) return false;
  avg_time = t;
  return launch_into(y_dev.p, acc ? 1.0 : 0.0) && ok(bsp_device_sync(), "bsp_device_sync");
}

bool to_i32(const int64_t *src, size_t n, std::vector<int32_t> &dst) {
  dst.resize(n);
  for (size_t i = 0; i < n; ++i) {
    if (src[i] < INT32_MIN || src[i] > INT32_MAX) {
      fprintf(stderr, "index %zu does not fit in int32\n", i);
      return false;
    }
    dst[i] = (int32_t)src[i];
  }
  return true;
}

// y on the device: the caller's values when accumulating, else zero-filled.
template <typename T>
bool y_init(Dev &y, const T *h, size_t n, bool acc = g_accumulate) {
  if (acc) return y.upload(h, n);
  std::vector<T> z(n, T(0));
  return y.upload(z.data(), n);
}

bool csr_f64(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz, double *values, double *x,
             double *out, int warm, int repeat, double &avg_time, int32_t algo, bool acc) {
  Dev rp, ci, va, xd, yd;
  if (!rp.upload(rowPtr, (size_t)rows + 1) || !ci.upload(colIdx, nnz) || !va.upload(values, nnz) ||
      !xd.upload(x, cols) || !y_init(yd, out, rows, acc))
    return false;
  const bool done = run_result(
      warm, repeat, yd, sizeof(double) * rows, avg_time,
      [&](void *y, double beta) {
        return ok(bsp_csr_spmv(rows, cols, nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.p, BSP_F64, xd.p, y, 1.0,
                               beta, algo, 0, nullptr),
                  "bsp_csr_spmv");
      },
      acc);
  return done && yd.download(out, rows);
}

}  // namespace

extern "C" void bsp_compat_set_accumulate(int on) { g_accumulate = on != 0; }
extern "C" int bsp_compat_get_accumulate(void) { return g_accumulate ? 1 : 0; }

int spmv_fp64_warpper(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz, double *values,
                      double *x, double *outvalues, int repeat, double &avg_time) {
  return csr_f64(rowPtr, colIdx, rows, cols, nnz, values, x, outvalues, 10, repeat, avg_time, BSP_CSR_AUTO,
                 g_accumulate)
             ? 0
             : 1;
}

int spmv_fp64_balance_warpper(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz,
                              double *values, double *x, double *outvalues, int repeat, double &avg_time) {
  return csr_f64(rowPtr, colIdx, rows, cols, nnz, values, x, outvalues, 10, repeat, avg_time, BSP_CSR_MERGE,
                 g_accumulate)
             ? 0
             : 1;
}

void MySpmvWithPre(int *rowPtr, int *colIdx, int rows, int cols, int nnz, float *values, float *x,
                   float *outvalues) {
  Dev rp, ci, va, xd, yd;
  if (!rp.upload(rowPtr, (size_t)rows + 1) || !ci.upload(colIdx, nnz) || !va.upload(values, nnz) ||
      !xd.upload(x, cols) || !yd.alloc(sizeof(float) * rows))
    return;
  if (ok(bsp_csr_spmv(rows, cols, nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.p, BSP_F32, xd.p, yd.p, 1.0, 0.0,
                      BSP_CSR_AUTO, 0, nullptr),
         "bsp_csr_spmv"))
    yd.download(outvalues, rows);
}

void MySpmvWithPrefp16(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz, float *values,
                       float *x, float *outvalues) {
  std::vector<half> hv(nnz), hx(cols), hy(rows);
  for (int32_t i = 0; i < nnz; ++i) hv[i] = __float2half(values[i]);
  for (int32_t i = 0; i < cols; ++i) hx[i] = __float2half(x[i]);
  Dev rp, ci, va, xd, yd;
  if (!rp.upload(rowPtr, (size_t)rows + 1) || !ci.upload(colIdx, nnz) || !va.upload(hv.data(), nnz) ||
      !xd.upload(hx.data(), cols) || !yd.alloc(sizeof(half) * rows))
    return;
  if (!ok(bsp_csr_spmv(rows, cols, nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.p, BSP_F16, xd.p, yd.p, 1.0, 0.0,
                       BSP_CSR_AUTO, 0, nullptr),
          "bsp_csr_spmv") ||
      !yd.download(hy.data(), rows))
    return;
  for (int32_t i = 0; i < rows; ++i) outvalues[i] = __half2float(hy[i]);
}

void MySpmvWithPrefp64(int64_t *rowPtr, int64_t *colIdx, int64_t rows, int64_t cols, int64_t nnz, double *values,
                       double *x, double *outvalues) {
  if (rows > INT32_MAX || cols > INT32_MAX || nnz > INT32_MAX) {
    fprintf(stderr, "MySpmvWithPrefp64: sizes must fit in int32\n");
    return;
  }
  std::vector<int32_t> rp, ci;
  if (!to_i32(rowPtr, (size_t)rows + 1, rp) || !to_i32(colIdx, (size_t)nnz, ci)) return;
  double t = 0;
  csr_f64(rp.data(), ci.data(), (int32_t)rows, (int32_t)cols, (int32_t)nnz, values, x, outvalues, 0, 0, t,
          BSP_CSR_AUTO, false);
}

int amgT_spmv_fp64(int32_t *hA_csrOffsets, int32_t *hA_columns, double *hA_values, double *hX, double *hY,
                   int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz, int repeat, double &avg_time) {
  Dev rp, ci, va, xd, yd;
  if (!rp.upload(hA_csrOffsets, (size_t)A_num_rows + 1) || !ci.upload(hA_columns, A_nnz) ||
      !va.upload(hA_values, A_nnz) || !xd.upload(hX, A_num_cols) || !y_init(yd, hY, A_num_rows))
    return 1;
  bsp_bsr m;
  if (!ok(bsp_csr2bsr(A_num_rows, A_num_cols, A_nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.as<double>(), 4, &m,
                      nullptr),
          "bsp_csr2bsr"))
    return 1;
  const bool done = run_result(5, repeat, yd, sizeof(double) * A_num_rows, avg_time, [&](void *y, double beta) {
    return ok(bsp_bsr_spmv(&m, xd.as<double>(), static_cast<double *>(y), 1.0, beta, BSP_BSR_AUTO, nullptr),
              "bsp_bsr_spmv");
  });
  bsp_bsr_free(&m);
  return done && yd.download(hY, A_num_rows) ? 0 : 1;
}

namespace {
int dbsr_call(dbsrMat *h, double *hX, double *hY, int32_t warmup, int32_t repeat, double &avg_time) {
  if (!h || h->blocknnz < 0 || h->blocknnz % 16 != 0) {
    fprintf(stderr, "amgT_spmv_fp64_dbsr: bad dbsrMat\n");
    return 1;
  }
  const int32_t nb = h->blocknnz / 16;
  Dev bp, ci, bv, bm, xd, yd;
  std::vector<uint16_t> map((size_t)nb + 1, 0xFFFFu);  // all entries live when the caller has no bitmap
  if (h->blcMap)
    for (int32_t i = 0; i < nb; ++i) map[i] = h->blcMap[i];
  if (!bp.upload(h->blcPtr, (size_t)h->blc_row + 1) || !ci.upload(h->colIdx, (size_t)h->blocknnz) ||
      !bv.upload(h->blcVal, (size_t)h->blocknnz) || !bm.upload(map.data(), map.size()) || !xd.upload(hX, h->col) ||
      !y_init(yd, hY, h->row))
    return 1;
  bsp_dbsr d;
  memset(&d, 0, sizeof(d));
  d.row = h->row;
  d.col = h->col;
  d.nnz = h->nnz;
  d.blc_row = h->blc_row;
  d.blc_col = h->blc_col;
  d.blc_num = nb;
  d.stand = h->stand;
  d.avg_nnz = h->avg_nnz;
  d.blcPtr = bp.as<int32_t>();
  d.colIdx = ci.as<int32_t>();
  d.blcVal = bv.as<double>();
  d.blcMap = bm.as<uint16_t>();
  d.blocknnz = h->blocknnz;
  d.warpnum = h->warpnum;
  const bool done = run_result(warmup, repeat, yd, sizeof(double) * h->row, avg_time, [&](void *y, double beta) {
    return ok(bsp_dbsr_spmv(&d, xd.as<double>(), static_cast<double *>(y), 1.0, beta, 1, nullptr),
              "bsp_dbsr_spmv");
  });
  return done && yd.download(hY, h->row) ? 0 : 1;
}
}  // namespace

int amgT_spmv_fp64_dbsr(dbsrMat *dbsr, double *hX, double *hY, int32_t warmup, int32_t repeat, double &avg_time) {
  return dbsr_call(dbsr, hX, hY, warmup, repeat, avg_time);
}

int amgT_spmv_fp64_dbsr_balance(dbsrMat *dbsr, double *hX, double *hY, int32_t warmup, int32_t repeat,
                                double &avg_time) {
  return dbsr_call(dbsr, hX, hY, warmup, repeat, avg_time);
}

void bcsr_spmv_fp64(int64_t *hA_csrOffsets, int64_t *hA_columns, double *hA_values32, double *hX32,
                    double *hY32, int64_t A_num_rows, int64_t A_num_cols, int64_t A_nnz, int repeat) {
  if (A_num_rows > INT32_MAX || A_num_cols > INT32_MAX || A_nnz > INT32_MAX) {
    fprintf(stderr, "bcsr_spmv_fp64: sizes must fit in int32\n");
    return;
  }
  const int32_t rows = (int32_t)A_num_rows, cols = (int32_t)A_num_cols, nnz = (int32_t)A_nnz;
  std::vector<int32_t> rp, ci;
  if (!to_i32(hA_csrOffsets, (size_t)rows + 1, rp) || !to_i32(hA_columns, (size_t)nnz, ci)) return;
  Dev drp, dci, dva, xd, yd;
  if (!drp.upload(rp.data(), rp.size()) || !dci.upload(ci.data(), ci.size()) || !dva.upload(hA_values32, nnz) ||
      !xd.upload(hX32, cols) || !y_init(yd, hY32, rows))
    return;
  bsp_bcsr b;
  if (!ok(bsp_csr2bcsr(rows, cols, nnz, drp.as<int32_t>(), dci.as<int32_t>(), dva.as<double>(), 3, 3, 0, &b,
                       nullptr),
          "bsp_csr2bcsr"))
    return;
  for (int i = 0; i < repeat; ++i) {  // the reference prints one time per launch
    double t = 0;
    const bool done = run_result(0, 1, yd, sizeof(double) * rows, t, [&](void *y, double beta) {
      return ok(bsp_bcsr_spmv(&b, xd.as<double>(), static_cast<double *>(y), 1.0, beta, nullptr), "bsp_bcsr_spmv");
    });
    if (!done) break;
    printf("bcsr time: %.2f us\n", t);
  }
  if (repeat <= 0) {
    double t = 0;
    run_result(0, 0, yd, sizeof(double) * rows, t, [&](void *y, double beta) {
      return ok(bsp_bcsr_spmv(&b, xd.as<double>(), static_cast<double *>(y), 1.0, beta, nullptr), "bsp_bcsr_spmv");
    });
  }
  bsp_bcsr_free(&b);
  yd.download(hY32, rows);
}

void spmv_all(char *filename, double *csrValA, int *csrRowPtrA, int *csrColIdxA, double *X_val, double *Y_val,
              int *order_rid, int rowA, int colA, int nnzA, int NUM, double threshold, int block_longest,
              double &avg_time) {
  (void)filename;
  (void)NUM;
  Dev rp, ci, va, xd, yd;
  if (!rp.upload(csrRowPtrA, (size_t)rowA + 1) || !ci.upload(csrColIdxA, nnzA) || !va.upload(csrValA, nnzA) ||
      !xd.upload(X_val, colA) || !y_init(yd, Y_val, rowA))
    return;
  bsp_dasp d;
  if (!ok(bsp_csr2dasp(rowA, colA, nnzA, rp.as<int32_t>(), ci.as<int32_t>(), va.as<double>(), threshold,
                       block_longest, &d, nullptr),
          "bsp_csr2dasp"))
    return;
  const bool done = run_result(10, 100, yd, sizeof(double) * rowA, avg_time, [&](void *y, double beta) {
    return ok(bsp_dasp_spmv(&d, xd.as<double>(), static_cast<double *>(y), 1.0, beta, 1, nullptr), "bsp_dasp_spmv");
  });
  if (done && yd.download(Y_val, rowA) && rowA > 0)
    ok(bsp_memcpy_d2h(order_rid, d.order_rid, sizeof(int32_t) * rowA), "bsp_memcpy_d2h");
  bsp_dasp_free(&d);
}

namespace {
// Fraction of the 16x16 tiles' entries that are nonzero (host CSR).
double tile_fill(const int *rowPtr, const int *colIdx, int rows, int64_t nnz) {
  int64_t tiles = 0;
  std::vector<int> tc;
  for (int r0 = 0; r0 < rows; r0 += 16) {
    tc.clear();
    for (int r = r0; r < std::min(rows, r0 + 16); ++r)
      for (int j = rowPtr[r]; j < rowPtr[r + 1]; ++j) tc.push_back(colIdx[j] >> 4);
    std::sort(tc.begin(), tc.end());
    tiles += std::unique(tc.begin(), tc.end()) - tc.begin();
  }
  return tiles ? (double)nnz / ((double)tiles * 256.0) : 0.0;
}
}  // namespace

void smatSpmmfp16(int *rowPtr, int *colIdx, int row, int col, int n, int nnz, float *values, float *outvalues) {
  if (row < 0 || col < 0 || n < 0 || nnz < 0) return;
  std::vector<half> ones((size_t)col * n, __float2half(1.0f));
  Dev rp, ci, Bd, Cd;
  if (!rp.upload(rowPtr, (size_t)row + 1) || !ci.upload(colIdx, nnz) || !Bd.upload(ones.data(), ones.size()) ||
      !Cd.alloc(sizeof(float) * (size_t)row * n))
    return;
  double t = -1;
  if (n % 32 == 0 && tile_fill(rowPtr, colIdx, row, nnz) >= 0.25) {
    // dense 16x16 tiles: the tensor-core tile path
    std::vector<double> v64(values, values + nnz);
    Dev va;
    if (!va.upload(v64.data(), v64.size())) return;
    bsp_smat m;
    if (!ok(bsp_smat_create(row, col, nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.as<double>(), BSP_F16, &m,
                            nullptr),
            "bsp_smat_create"))
      return;
    t = timed(1, 1, [&] {
      return ok(bsp_smat_spmm(&m, Bd.p, n, n, Cd.as<float>(), n, 1.0f, 0.0f, nullptr), "bsp_smat_spmm");
    });
    if (t >= 0) ok(bsp_smat_check(&m, nullptr), "bsp_smat_check");
    bsp_smat_free(&m);
  } else {
    // scattered nonzeros: row-split CSR SpMM
    std::vector<half> hv(nnz);
    for (int i = 0; i < nnz; ++i) hv[i] = __float2half(values[i]);
    Dev va;
    if (!va.upload(hv.data(), hv.size())) return;
    bsp_spmm_plan p;
    if (!ok(bsp_spmm_plan_create(row, nnz, rp.as<int32_t>(), 256, &p, nullptr), "bsp_spmm_plan_create")) return;
    Dev ws;
    const size_t wsb = bsp_spmm_plan_workspace(&p, n);
    if (ws.alloc(wsb))
      t = timed(1, 1, [&] {
        return ok(bsp_spmm_csr_planned(&p, col, nnz, rp.as<int32_t>(), ci.as<int32_t>(), va.p, BSP_F16, Bd.p, n, n,
                                       Cd.as<float>(), n, 1.0f, 0.0f, ws.p, wsb, nullptr),
                  "bsp_spmm_csr_planned");
      });
    bsp_spmm_plan_free(&p);
  }
  if (t < 0) return;
  printf("smat time: %.2f us\n", t);
  Cd.download(outvalues, (size_t)row * n);
}
