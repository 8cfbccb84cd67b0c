// Drop-in for the part of the fast_matrix_market header that the reference's
// bench drivers use (read_matrix_market_triplet + read_options; called from
// read_triplet_file, bench/spmvfp64.cpp:37-44, bench/spmvfp16.cpp:32-39,
// bench/spmmfp16.cpp:32-39, bench/blockinfo.cpp:39-45).  The reference's
// CMakeLists.txt:15-21 fetches that library unpinned from its main branch;
// with this directory on the include path instead, the drivers compile
// unchanged and read through libbspmv's Matrix Market parser
// (bsp_mtx_read_buffer, include/bsp.h): link with -lbspmv.
//
// read_options mirrors the library's defaults: symmetric files are
// generalised (generalize_symmetry = true), each diagonal entry of such a
// file getting an explicit zero partner (ExtraZeroElement) or a copy of
// itself (DuplicateElement).  chunk_size_bytes, parallel_ok and num_threads
// are accepted; num_threads (0 = all host threads) sets the parse threads.
//
// Two drivers open a fixed path on the reference author's machine
// (bench/spmvfp16.cpp:41, bench/spmmfp16.cpp:37); when the stream they pass
// did not open and BSP_MTX_FILE is set, that file is read instead.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <istream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <vector>

#include "bsp.h"

namespace fast_matrix_market {

struct read_options {
  enum { ExtraZeroElement, DuplicateElement } generalize_coordinate_diagnonal_values = ExtraZeroElement;
  int64_t chunk_size_bytes = 2 << 20;
  bool generalize_symmetry = true;
  bool parallel_ok = true;
  int num_threads = 0;
};

struct fmm_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

namespace detail {

inline std::string slurp(std::istream &in) {
  std::ifstream redirect;
  std::istream *src = &in;
  if (!in.good())
    if (const char *p = std::getenv("BSP_MTX_FILE")) {
      redirect.open(p, std::ios::binary);
      src = &redirect;
    }
  if (!src->good()) throw fmm_error("cannot read the Matrix Market stream");
  return std::string(std::istreambuf_iterator<char>(*src), std::istreambuf_iterator<char>());
}

struct handle {
  bsp_mtx m = nullptr;
  ~handle() {
    if (m) bsp_mtx_free(m);
  }
};

}  // namespace detail

template <typename IT, typename VT, typename DIM>
void read_matrix_market_triplet(std::istream &in, DIM &nrows, DIM &ncols, std::vector<IT> &rows,
                                std::vector<IT> &cols, std::vector<VT> &vals, const read_options &options = {}) {
  const std::string text = detail::slurp(in);
  int32_t flags = 0;
  if (!options.generalize_symmetry)
    flags |= BSP_MTX_NO_EXPAND;
  else if (options.generalize_coordinate_diagnonal_values == read_options::ExtraZeroElement)
    flags |= BSP_MTX_DIAG_ZERO;
  else
    flags |= BSP_MTX_DIAG_DUPLICATE;
  const int32_t threads = options.parallel_ok ? (int32_t)options.num_threads : 1;
  detail::handle h;
  if (bsp_mtx_read_buffer(text.data(), text.size(), flags, threads, &h.m) != BSP_OK)
    throw fmm_error(bsp_last_error());
  bsp_mtx_info info;
  bsp_mtx_get_info(h.m, &info);
  std::vector<int32_t> r((size_t)info.nnz), c((size_t)info.nnz);
  std::vector<double> v((size_t)info.nnz);
  if (bsp_mtx_triplets(h.m, r.data(), c.data(), v.data()) != BSP_OK) throw fmm_error(bsp_last_error());
  nrows = (DIM)info.rows;
  ncols = (DIM)info.cols;
  rows.assign(r.begin(), r.end());
  cols.assign(c.begin(), c.end());
  vals.resize(v.size());
  for (size_t k = 0; k < v.size(); ++k) vals[k] = (VT)v[k];
}

}  // namespace fast_matrix_market
