// Minimal stand-in for the fast_matrix_market header the reference's bench
// drivers include (fetched from the network by its CMakeLists.txt:15-21, not
// available here).  TEST INFRASTRUCTURE ONLY: it lets oracle/Makefile compile
// the reference's bench/blockinfo.cpp unchanged as an oracle of its block
// statistics, independent of the library's own reader (the bench drivers
// linked against libbspmv_compat use the library's drop-in header instead).
// Reads Matrix Market coordinate files (real / integer / pattern, general or
// symmetric) into triplet vectors, 1-based -> 0-based.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <istream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace fast_matrix_market {

struct read_options {
  int64_t chunk_size_bytes = 1 << 20;
};

template <typename IT, typename VT, typename DIM>
void read_matrix_market_triplet(std::istream &in0, DIM &nrows, DIM &ncols, std::vector<IT> &rows,
                                std::vector<IT> &cols, std::vector<VT> &vals, const read_options & = {}) {
  std::istream &in = in0;
  std::string line;
  if (!std::getline(in, line) || line.rfind("%%MatrixMarket", 0) != 0) throw std::runtime_error("not a MatrixMarket file");
  const bool pattern = line.find("pattern") != std::string::npos;
  const bool symmetric = line.find("symmetric") != std::string::npos;
  while (std::getline(in, line))
    if (!line.empty() && line[0] != '%') break;
  std::istringstream hdr(line);
  int64_t r, c, n;
  hdr >> r >> c >> n;
  nrows = (DIM)r;
  ncols = (DIM)c;
  rows.clear();
  cols.clear();
  vals.clear();
  for (int64_t k = 0; k < n; ++k) {
    int64_t i, j;
    double v = 1.0;
    in >> i >> j;
    if (!pattern) in >> v;
    rows.push_back((IT)(i - 1));
    cols.push_back((IT)(j - 1));
    vals.push_back((VT)v);
    if (symmetric && i != j) {
      rows.push_back((IT)(j - 1));
      cols.push_back((IT)(i - 1));
      vals.push_back((VT)v);
    }
  }
}

}  // namespace fast_matrix_market
