// Runs the reference's DASP kernels (dasp_spmv2<1> + longPart_sum,
// src/dasp.cu:381-812, compiled for sm_100a) on the B200 with the exact
// arguments its spmv_all (src/dasp.cu:814) hands to the first launch, as
// recorded by oracle/_ref/dasp_capture, and times them with CUDA events.
// TEST INFRASTRUCTURE ONLY (oracle/_ref/ref_dasp_time, run by
// tests/test_ref_gpu_kernels.py).  spmv_all itself synchronises after every
// launch and times with the host clock; here the two launches of a product
// run back to back.
//
//   ref_dasp_time <capture.bin> <y_out.bin> <reps>
//   y_out.bin: y (f64, rows in order_rid order) after one product on y = 0
//   stdout: {"dasp_spmv2+longPart_sum": median us per product}
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

template <int rowloop>
__global__ void dasp_spmv2(double *dX_val, double *dY_val, double *dlongA_val, int *dlongA_cid, double *dwarp_val,
                           int *dlongA_rpt, int row_long, double *dregA_val, int *dregA_cid, int *dblockA_ptr,
                           int row_block, int blocknum, double *dirregA_val, int *dirregA_cid, int *dirregA_rpt,
                           double *dshort_val, int *dshort_cid, int short_row_1, int common_13, int short_row_34,
                           int short_row_2, int offset_reg, int offset_short1, int offset_short13, int offset_short34,
                           int offset_short22, int fill0_nnz_short13, int fill0_nnz_short34);
__global__ void longPart_sum(int *dlongA_rpt, double *dwarp_val, double *dY_val, int row_long);

#define CK(x)                                                                     \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) {                                                      \
      fprintf(stderr, "%s:%d %s -> %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      exit(4);                                                                    \
    }                                                                             \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 4) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  std::map<std::string, std::vector<char>> rec;
  for (;;) {
    int32_t nl;
    if (fread(&nl, 4, 1, f) != 1) break;
    std::string name((size_t)nl, '\0');
    int64_t nb;
    if (fread(&name[0], 1, nl, f) != (size_t)nl || fread(&nb, 8, 1, f) != 1) return 3;
    std::vector<char> d((size_t)nb);
    if (nb && fread(d.data(), 1, nb, f) != (size_t)nb) return 3;
    rec[name] = std::move(d);
  }
  fclose(f);
  const int reps = atoi(argv[3]);
  auto I = [&](const char *n) -> int {
    auto it = rec.find(std::string("int:") + n);
    if (it == rec.end()) {
      fprintf(stderr, "missing int %s\n", n);
      exit(5);
    }
    return *reinterpret_cast<const int32_t *>(it->second.data());
  };
  std::map<std::string, void *> dev;
  auto A = [&](const char *n) -> void * {
    const std::string key = std::string("arr:") + n;
    auto d = dev.find(key);
    if (d != dev.end()) return d->second;
    auto it = rec.find(key);
    void *p = nullptr;
    const size_t nb = it == rec.end() ? 0 : it->second.size();
    CK(cudaMalloc(&p, nb < 64 ? 64 : nb));
    CK(cudaMemset(p, 0, nb < 64 ? 64 : nb));
    if (nb) CK(cudaMemcpy(p, it->second.data(), nb, cudaMemcpyHostToDevice));
    dev[key] = p;
    return p;
  };
  double *X = (double *)A("dX_val"), *Y = (double *)A("dY_val");
  const int row_long = I("row_long");
  const int grid = I("grid_all"), block = I("block_all");
  const int grid_sum = row_long ? I("grid_longsum") : 0;
  const size_t ybytes = rec["arr:dY_val"].size();
  auto product = [&] {
    dasp_spmv2<1><<<grid, block>>>(X, Y, (double *)A("long_val"), (int *)A("long_cid"), (double *)A("warp_val"),
                                   (int *)A("long_ptr_warp"), row_long, (double *)A("reg_val"), (int *)A("reg_cid"),
                                   (int *)A("block_ptr"), I("row_block"), I("blocknum"), (double *)A("irreg_val"),
                                   (int *)A("irreg_cid"), (int *)A("irreg_rpt"), (double *)A("short_val"),
                                   (int *)A("short_cid"), I("short_row_1"), I("common_13"), I("short_row_34"),
                                   I("short_row_2"), I("offset_reg"), I("offset_short1"), I("offset_short13"),
                                   I("offset_short34"), I("offset_short22"), I("fill0_nnz_short13"),
                                   I("fill0_nnz_short34"));
    if (row_long) longPart_sum<<<grid_sum, block>>>((int *)A("long_ptr_warp"), (double *)A("warp_val"), Y, row_long);
  };
  // every device array is created before timing
  product();
  CK(cudaDeviceSynchronize());
  CK(cudaMemset(Y, 0, ybytes));
  product();
  CK(cudaDeviceSynchronize());
  std::vector<char> h(ybytes);
  CK(cudaMemcpy(h.data(), Y, ybytes, cudaMemcpyDeviceToHost));
  FILE *o = fopen(argv[2], "wb");
  if (!o) return 3;
  fwrite(h.data(), 1, ybytes, o);
  fclose(o);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  for (int i = 0; i < 5; ++i) product();
  CK(cudaEventRecord(a));
  for (int i = 0; i < reps; ++i) product();
  CK(cudaEventRecord(b));
  CK(cudaEventSynchronize(b));
  CK(cudaGetLastError());
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, a, b));
  printf("{\"dasp_spmv2+longPart_sum\": %.3f}\n", 1e3 * ms / reps);
  return 0;
}
