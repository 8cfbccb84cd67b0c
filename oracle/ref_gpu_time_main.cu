// Runs the reference's own SpMV kernels, compiled for sm_100a from their
// sources, on arrays given in a file, and reports each kernel's result and
// CUDA-event time.  TEST INFRASTRUCTURE ONLY (oracle/_ref/ref_amgt_time and
// oracle/_ref/ref_csr_time, run by tests/test_ref_gpu_kernels.py): the
// kernels are called directly with the launch shapes their wrappers use
// (src/amgT.cu:1355-1488, src/csrspmv.cu:104-195), without the wrappers'
// host copies and per-launch synchronisation.
//
//   ref_amgt_time <in.bin> <out.bin> <reps>
//     in.bin: int32 row, col, blc_row, blc_col, blc_num, warpnum; blcPtr,
//             blcIdx (int32), blcVal (f64, 16 per block), blcMap (uint16),
//             rowPtrbyWarp, rowIdxbyWarp (int32), x (f64)
//   ref_csr_time <in.bin> <out.bin> <reps> [flush_mb]
//     in.bin: int32 rows, cols, nnz; rowPtr, colIdx (int32), values, x (f64)
//   out.bin: for every kernel, its y (f64) after one launch on y = 0.
//   stdout: one JSON object {kernel: median microseconds per launch}.
// A flush_mb > 0 writes that many MB between timed launches (L2 flush) and
// times each launch alone.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#ifdef REF_AMGT
__global__ void bsr_spmv_tc_fp64(int *d_blcPtr, int *d_blcCid, double *d_blcVal, double *d_x, double *d_y,
                                 int blc_row, int blc_col, int row, int col, double alpha);
__global__ void bsr_spmv_cc_fp64(int *d_blcPtr, int *d_blcCid, unsigned short *d_blcMap, double *d_blcVal,
                                 double *d_x, double *d_y, int blc_row, int blc_col, int row, int col, double alpha);
__global__ void bsr_spmv_balanced_tc_fp64(int *rowPtrbyWarp, int *rowIdxbyWarp, int warp_num, int *d_blcPtr,
                                          int *d_blcCid, double *d_blcVal, double *d_x, double *d_y, int blc_row,
                                          int blc_col, int row, int col, double alpha);
__global__ void bsr_spmv_balanced_cc_fp64(int *rowPtrbyWarp, int *rowIdxbyWarp, int warp_num, int *d_blcPtr,
                                          int *d_blcCid, unsigned short *d_blcMap, double *d_blcVal, double *d_x,
                                          double *d_y, int blc_row, int blc_col, int row, int col, double alpha);
#endif
#ifdef REF_CSR
__global__ void spmv_fp64(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t nnz, double *values, double *x,
                          double *outvalues);
__global__ void get_rowPtrbyWarp_csr(int *d_blcPtr, int *rowPtrbyWarp, int blc_row);
__global__ void get_rowIdxbyWarp_csr(int *rowPtrbyWarp, int *rowIdxbyWarp, int blc_row);
__global__ void spmv_fp64_balance(int32_t *rowPtr, int32_t *rowPtrbyWarp, int32_t *colIdx, int32_t *rowIdxbyWarp,
                                  int32_t rows, int32_t nnz, int32_t warp_num, double *values, double *x, double *d_y);
#endif

#define CK(x)                                                                     \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) {                                                      \
      fprintf(stderr, "%s:%d %s -> %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      exit(4);                                                                    \
    }                                                                             \
  } while (0)

template <typename T>
static T *upload(FILE *f, int64_t n) {
  std::vector<T> h((size_t)std::max<int64_t>(n, 1));
  if (n > 0 && fread(h.data(), sizeof(T), (size_t)n, f) != (size_t)n) {
    fprintf(stderr, "short input\n");
    exit(3);
  }
  T *d = nullptr;
  CK(cudaMalloc(&d, sizeof(T) * h.size()));
  CK(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return d;
}

struct Timer {
  void *flush = nullptr;
  size_t flush_bytes = 0;
  // median microseconds of `reps` launches of fn (each alone when flushing,
  // else the mean of one back-to-back run of reps launches)
  template <typename F>
  double time(F fn, int reps) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (int i = 0; i < 5; ++i) fn();
    CK(cudaDeviceSynchronize());
    std::vector<float> t;
    if (flush_bytes) {
      for (int i = 0; i < reps; ++i) {
        CK(cudaMemsetAsync(flush, i & 0xff, flush_bytes));
        CK(cudaEventRecord(a));
        fn();
        CK(cudaEventRecord(b));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        t.push_back(ms);
      }
    } else {
      CK(cudaEventRecord(a));
      for (int i = 0; i < reps; ++i) fn();
      CK(cudaEventRecord(b));
      CK(cudaEventSynchronize(b));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, a, b));
      t.push_back(ms / reps);
    }
    CK(cudaGetLastError());
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(t.begin(), t.end());
    return 1e3 * t[t.size() / 2];
  }
};

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  FILE *f = fopen(argv[1], "rb");
  FILE *o = fopen(argv[2], "wb");
  if (!f || !o) return 3;
  const int reps = atoi(argv[3]);
  Timer T;
  if (argc > 4 && atoi(argv[4]) > 0) {
    T.flush_bytes = (size_t)atoi(argv[4]) << 20;
    CK(cudaMalloc(&T.flush, T.flush_bytes));
  }
  std::vector<std::pair<std::string, double>> out;
  auto dump = [&](const double *dy, int64_t n) {
    std::vector<double> h((size_t)n);
    CK(cudaMemcpy(h.data(), dy, sizeof(double) * n, cudaMemcpyDeviceToHost));
    fwrite(h.data(), sizeof(double), (size_t)n, o);
  };
#ifdef REF_AMGT
  int32_t hd[6];
  if (fread(hd, 4, 6, f) != 6) return 3;
  const int row = hd[0], col = hd[1], blc_row = hd[2], blc_col = hd[3], blc_num = hd[4], warpnum = hd[5];
  int *blcPtr = upload<int>(f, blc_row + 1);
  int *blcIdx = upload<int>(f, blc_num);
  double *blcVal = upload<double>(f, (int64_t)blc_num * 16);
  unsigned short *blcMap = upload<unsigned short>(f, blc_num);
  int *rpw = upload<int>(f, blc_row + 1);
  int *riw = upload<int>(f, warpnum);
  double *x = upload<double>(f, col);
  double *y = nullptr;
  CK(cudaMalloc(&y, sizeof(double) * row));
  const int threads = 32 * 4;  // WARP_SIZE * WARP_NUM_SPMV (include/common.h:8)
  const int blocks_b = (warpnum + 3) / 4, blocks = (blc_row + 3) / 4;
  auto tc = [&] { bsr_spmv_tc_fp64<<<blocks, threads>>>(blcPtr, blcIdx, blcVal, x, y, blc_row, blc_col, row, col, 1.0); };
  auto cc = [&] {
    bsr_spmv_cc_fp64<<<blocks, threads>>>(blcPtr, blcIdx, blcMap, blcVal, x, y, blc_row, blc_col, row, col, 1.0);
  };
  auto btc = [&] {
    bsr_spmv_balanced_tc_fp64<<<blocks_b, threads>>>(rpw, riw, warpnum, blcPtr, blcIdx, blcVal, x, y, blc_row,
                                                     blc_col, row, col, 1.0);
  };
  auto bcc = [&] {
    bsr_spmv_balanced_cc_fp64<<<blocks_b, threads>>>(rpw, riw, warpnum, blcPtr, blcIdx, blcMap, blcVal, x, y,
                                                     blc_row, blc_col, row, col, 1.0);
  };
  auto run = [&](const char *name, auto fn) {
    CK(cudaMemset(y, 0, sizeof(double) * row));
    fn();
    CK(cudaDeviceSynchronize());
    dump(y, row);
    out.push_back({name, T.time(fn, reps)});
  };
  run("bsr_spmv_tc_fp64", tc);
  run("bsr_spmv_cc_fp64", cc);
  run("bsr_spmv_balanced_tc_fp64", btc);
  run("bsr_spmv_balanced_cc_fp64", bcc);
#endif
#ifdef REF_CSR
  int32_t hd[3];
  if (fread(hd, 4, 3, f) != 3) return 3;
  const int rows = hd[0], cols = hd[1], nnz = hd[2];
  int *rp = upload<int>(f, rows + 1);
  int *ci = upload<int>(f, nnz);
  double *va = upload<double>(f, nnz);
  double *x = upload<double>(f, cols);
  double *y = nullptr;
  CK(cudaMalloc(&y, sizeof(double) * rows));
  (void)cols;
  // the balanced kernel's chunk map, built by the reference's own kernels
  // (the wrapper's thrust scan done on the host here)
  int *rpw = nullptr;
  CK(cudaMalloc(&rpw, sizeof(int) * (rows + 1)));
  CK(cudaMemset(rpw, 0, sizeof(int) * (rows + 1)));
  const int threads = 4 * 32;
  const int blocks = (rows + threads - 1) / threads;
  get_rowPtrbyWarp_csr<<<blocks, threads>>>(rp, rpw, rows);
  CK(cudaDeviceSynchronize());
  std::vector<int> h((size_t)rows + 1);
  CK(cudaMemcpy(h.data(), rpw, sizeof(int) * (rows + 1), cudaMemcpyDeviceToHost));
  int acc = 0;
  for (int i = 0; i <= rows; ++i) {
    const int v = h[i];
    h[i] = acc;
    acc += v;
  }
  const int warpnum = h[rows];
  CK(cudaMemcpy(rpw, h.data(), sizeof(int) * (rows + 1), cudaMemcpyHostToDevice));
  int *riw = nullptr;
  CK(cudaMalloc(&riw, sizeof(int) * std::max(warpnum, 1)));
  get_rowIdxbyWarp_csr<<<blocks, threads>>>(rpw, riw, rows);
  CK(cudaDeviceSynchronize());
  const int blocks_b = (warpnum + threads - 1) / threads;
  auto scalar = [&] { spmv_fp64<<<blocks, threads>>>(rp, ci, rows, nnz, va, x, y); };
  auto balance = [&] { spmv_fp64_balance<<<blocks_b, threads>>>(rp, rpw, ci, riw, rows, nnz, warpnum, va, x, y); };
  auto run = [&](const char *name, auto fn) {
    CK(cudaMemset(y, 0, sizeof(double) * rows));
    fn();
    CK(cudaDeviceSynchronize());
    dump(y, rows);
    out.push_back({name, T.time(fn, reps)});
  };
  run("spmv_fp64", scalar);
  run("spmv_fp64_balance", balance);
#endif
  fclose(o);
  printf("{");
  for (size_t i = 0; i < out.size(); ++i) printf("%s\"%s\": %.3f", i ? ", " : "", out[i].first.c_str(), out[i].second);
  printf("}\n");
  return 0;
}
