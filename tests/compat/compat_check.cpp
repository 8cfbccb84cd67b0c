// Calls every function of benchsp_compat.hpp (the reference's operator names)
// on one matrix and writes each result to <dir>/out_<name>.bin for the Python
// test to compare with the CPU oracle.
//
//   compat_check <dir>
// <dir> holds meta.txt ("rows cols nnz dbsr_blc_row dbsr_blocknnz n") and raw
// little-endian arrays: rowptr.i32 colidx.i32 values.f64 x.f64 yin.f64,
// dbsr_blcPtr.i32 dbsr_colIdx.i32 dbsr_blcVal.f64 dbsr_blcMap.u16.
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "benchsp_compat.hpp"

static std::string g_dir;

template <typename T>
static std::vector<T> load(const char *name, size_t n) {
  std::vector<T> v(n);
  const std::string p = g_dir + "/" + name;
  FILE *f = fopen(p.c_str(), "rb");
  if (!f || fread(v.data(), sizeof(T), n, f) != n) {
    fprintf(stderr, "cannot read %s\n", p.c_str());
    exit(2);
  }
  fclose(f);
  return v;
}

template <typename T>
static void save(const char *name, const T *p, size_t n) {
  const std::string q = g_dir + "/out_" + name + ".bin";
  FILE *f = fopen(q.c_str(), "wb");
  if (!f || fwrite(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "cannot write %s\n", q.c_str());
    exit(2);
  }
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc != 2) return 2;
  g_dir = argv[1];
  int rows, cols, nnz, dbr, dbnnz, n;
  {
    const std::string p = g_dir + "/meta.txt";
    FILE *f = fopen(p.c_str(), "r");
    if (!f || fscanf(f, "%d %d %d %d %d %d", &rows, &cols, &nnz, &dbr, &dbnnz, &n) != 6) return 2;
    fclose(f);
  }
  auto rp = load<int32_t>("rowptr.i32", rows + 1);
  auto ci = load<int32_t>("colidx.i32", nnz);
  auto va = load<double>("values.f64", nnz);
  auto x = load<double>("x.f64", cols);
  auto yin = load<double>("yin.f64", rows);
  std::vector<double> y(rows);
  double t = 0;
  int bad = 0;

  bad |= spmv_fp64_warpper(rp.data(), ci.data(), rows, cols, nnz, va.data(), x.data(), y.data(), 3, t);
  save("spmv_fp64_warpper", y.data(), rows);
  bad |= spmv_fp64_balance_warpper(rp.data(), ci.data(), rows, cols, nnz, va.data(), x.data(), y.data(), 3, t);
  save("spmv_fp64_balance_warpper", y.data(), rows);

  std::vector<int64_t> rp64(rp.begin(), rp.end()), ci64(ci.begin(), ci.end());
  MySpmvWithPrefp64(rp64.data(), ci64.data(), rows, cols, nnz, va.data(), x.data(), y.data());
  save("MySpmvWithPrefp64", y.data(), rows);

  std::vector<float> vf(va.begin(), va.end()), xf(x.begin(), x.end()), yf(rows);
  MySpmvWithPrefp16(rp.data(), ci.data(), rows, cols, nnz, vf.data(), xf.data(), yf.data());
  save("MySpmvWithPrefp16", yf.data(), rows);
  MySpmvWithPre(rp.data(), ci.data(), rows, cols, nnz, vf.data(), xf.data(), yf.data());
  save("MySpmvWithPre", yf.data(), rows);

  bad |= amgT_spmv_fp64(rp.data(), ci.data(), va.data(), x.data(), y.data(), rows, cols, nnz, 3, t);
  save("amgT_spmv_fp64", y.data(), rows);

  auto bp = load<int32_t>("dbsr_blcPtr.i32", dbr + 1);
  auto bc = load<int32_t>("dbsr_colIdx.i32", dbnnz);
  auto bv = load<double>("dbsr_blcVal.f64", dbnnz);
  auto bm = load<uint16_t>("dbsr_blcMap.u16", dbnnz / 16);
  dbsrMat d{};
  d.row = rows;
  d.col = cols;
  d.nnz = nnz;
  d.blc_row = dbr;
  d.blc_num = dbnnz / 16;
  d.blcPtr = bp.data();
  d.colIdx = bc.data();
  d.blcVal = bv.data();
  d.blcMap = bm.data();
  d.blocknnz = dbnnz;
  bad |= amgT_spmv_fp64_dbsr(&d, x.data(), y.data(), 1, 3, t);
  save("amgT_spmv_fp64_dbsr", y.data(), rows);
  bad |= amgT_spmv_fp64_dbsr_balance(&d, x.data(), y.data(), 1, 3, t);
  save("amgT_spmv_fp64_dbsr_balance", y.data(), rows);

  bcsr_spmv_fp64(rp64.data(), ci64.data(), va.data(), x.data(), y.data(), rows, cols, nnz, 2);
  save("bcsr_spmv_fp64", y.data(), rows);

  std::vector<int> order(rows);
  char fname[8] = "unused";
  spmv_all(fname, va.data(), rp.data(), ci.data(), x.data(), y.data(), order.data(), rows, cols, nnz, 4, 0.75, 256,
           t);
  save("spmv_all", y.data(), rows);
  save("spmv_all_order", order.data(), rows);

  std::vector<float> C((size_t)rows * n);
  smatSpmmfp16(rp.data(), ci.data(), rows, cols, n, nnz, vf.data(), C.data());
  save("smatSpmmfp16", C.data(), C.size());

  bad |= cusparse_spmv_fp64(rp64.data(), ci64.data(), va.data(), x.data(), y.data(), rows, cols, nnz, 3, t);
  save("cusparse_spmv_fp64", y.data(), rows);
  cusparse_spmv_fp16_warpper(rp.data(), ci.data(), vf.data(), xf.data(), yf.data(), rows, cols, nnz);
  save("cusparse_spmv_fp16_warpper", yf.data(), rows);
  bad |= cusparse_spmv(rp.data(), ci64.data(), vf.data(), xf.data(), yf.data(), rows, cols, nnz);
  save("cusparse_spmv", yf.data(), rows);

  bsp_compat_set_accumulate(1);
  y = yin;
  bad |= spmv_fp64_warpper(rp.data(), ci.data(), rows, cols, nnz, va.data(), x.data(), y.data(), 2, t);
  save("accumulate_spmv_fp64_warpper", y.data(), rows);
  y = yin;
  bad |= amgT_spmv_fp64(rp.data(), ci.data(), va.data(), x.data(), y.data(), rows, cols, nnz, 2, t);
  save("accumulate_amgT_spmv_fp64", y.data(), rows);
  bsp_compat_set_accumulate(0);

  printf("compat_check done, status %d\n", bad);
  return bad ? 1 : 0;
}
