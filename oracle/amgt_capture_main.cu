// Runs the reference's own device CSR->BSR conversion (CSR2BSR_GPU and
// BSR_BALANCED_PREPROCESS_GPU, src/amgT.cu:1114-1200) on a GPU and writes
// the arrays it builds.  TEST INFRASTRUCTURE ONLY (oracle/_ref/amgt_capture,
// run by the GPU parity tests to pin the library's conversion).
//
//   amgt_capture <in.bin> <out.bin>     (in.bin as for dasp_capture)
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <string.h>
#include <string>
#include <vector>

#include "matrixFormat.hpp"

void CSR2BSR_GPU(bsrMAT *bsrmat, int32_t *hA_csrOffsets, int32_t *hA_columns, double *hA_values, double *hX,
                 double *hY, int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz);
void BSR_BALANCED_PREPROCESS_GPU(bsrMAT *bsrmat);

static FILE *g_o;
static void put(const char *name, const void *p, int64_t n) {
  const int32_t nl = (int32_t)strlen(name);
  fwrite(&nl, 4, 1, g_o);
  fwrite(name, 1, nl, g_o);
  fwrite(&n, 8, 1, g_o);
  if (n) fwrite(p, 1, n, g_o);
}
template <typename T>
static void put_dev(const char *name, const T *d, int64_t count) {
  std::vector<T> h(count > 0 ? count : 1);
  if (count > 0) cudaMemcpy(h.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost);
  put(name, h.data(), (int64_t)sizeof(T) * count);
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  int32_t rows, cols, nnz, bl;
  double th;
  if (fread(&rows, 4, 1, f) != 1 || fread(&cols, 4, 1, f) != 1 || fread(&nnz, 4, 1, f) != 1 ||
      fread(&th, 8, 1, f) != 1 || fread(&bl, 4, 1, f) != 1)
    return 4;
  std::vector<int32_t> rp(rows + 1), ci(nnz);
  std::vector<double> v(nnz), x(cols), y(rows, 0.0);
  if (fread(rp.data(), 4, rows + 1, f) != (size_t)rows + 1 || fread(ci.data(), 4, nnz, f) != (size_t)nnz ||
      fread(v.data(), 8, nnz, f) != (size_t)nnz || fread(x.data(), 8, cols, f) != (size_t)cols)
    return 5;
  fclose(f);
  bsrMAT m;
  CSR2BSR_GPU(&m, rp.data(), ci.data(), v.data(), x.data(), y.data(), rows, cols, nnz);
  const double stand = m.stand;  // BSR_BALANCED_PREPROCESS_GPU overwrites it with 12
  BSR_BALANCED_PREPROCESS_GPU(&m);
  if (cudaDeviceSynchronize() != cudaSuccess) return 7;
  g_o = fopen(argv[2], "wb");
  if (!g_o) return 6;
  const int32_t ints[6] = {m.row, m.col, m.nnz, m.blc_row, m.blc_col, m.blc_num};
  put("ints:row,col,nnz,blc_row,blc_col,blc_num", ints, sizeof(ints));
  put("f64:stand", &stand, 8);
  put("f64:avg_nnz", &m.avg_nnz, 8);
  put("int:warpnum", &m.warpnum, 4);
  put_dev("arr:blcPtr", m.blcPtr, (int64_t)m.blc_row + 1);
  put_dev("arr:blcIdx", m.blcIdx, m.blc_num);
  put_dev("arr:blcVal", m.blcVal, (int64_t)m.blc_num * 16);
  put_dev("arr:blcMap", m.blcMap, m.blc_num);
  put_dev("arr:rowPtrbyWarp", m.rowPtrbyWarp, (int64_t)m.blc_row + 1);
  put_dev("arr:rowIdxbyWarp", m.rowIdxbyWarp, m.warpnum);
  fclose(g_o);
  return cudaGetLastError() == cudaSuccess ? 0 : 8;
}
