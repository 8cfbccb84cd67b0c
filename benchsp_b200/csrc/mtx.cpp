// Matrix Market files: reader (host threads) and writer.
//
// The reference reads its inputs in the bench drivers through the
// third-party fast_matrix_market header (read_triplet_file,
// bench/spmvfp64.cpp:37-44; fetched unpinned from its main branch by
// CMakeLists.txt:15-21), then sorts the triplets by (row, col) with std::sort
// and counts rows into a CSR row pointer (bench/spmvfp64.cpp:56-86).  This
// file restates that pipeline as a library call:
//   * the file is mapped and cut into one byte range per thread at line
//     boundaries; a first pass counts each range's data lines, a second
//     parses them (std::from_chars: correctly rounded decimal -> double, as
//     fast_matrix_market's parser) straight into the triplet arrays at the
//     prefix offsets, so the triplets keep file order whatever the thread
//     count;
//   * a non-general file is expanded with one mirrored entry per off-diagonal
//     entry, appended in file order (negated for skew-symmetric), and with
//     BSP_MTX_DIAG_ZERO an explicit 0.0 mirror per diagonal entry, which is
//     fast_matrix_market's default element count for generalised symmetry;
//   * CSR: a row count + scatter of (col << 32 | triplet index) keys, then a
//     per-row sort of the keys, which orders by column and keeps triplet
//     order among equal (row, col); duplicates are kept, as the reference's
//     conversion keeps them (the order it gives equal keys is std::sort's,
//     i.e. unspecified; this one is stable).  Triplets that the parse found
//     already in (row, col) order (files written row by row) skip the sort;
//     on the device, triplets in (col, row) order (column-major files) skip
//     the first of the two sorts.
//     The device form (mtx_dev.cu) gives the same arrays.
#include <fcntl.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <charconv>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/bsp.h"

namespace bsp {
void set_error(const std::string &msg);
void clear_error();
bsp_status mtx_csr_device(int32_t rows, int32_t cols, int64_t nnz, const int32_t *r, const int32_t *c,
                          const double *v, bool sorted, bool col_sorted, int32_t *rowPtr, int32_t *colIdx,
                          double *values, cudaStream_t s);
}  // namespace bsp

struct bsp_mtx_s {
  bsp_mtx_info info{};
  std::unique_ptr<int32_t[]> r, c;  // triplets (info.nnz used)
  std::unique_ptr<double[]> v;
  bool sorted = false;               // already in (row, col) order
  bool col_sorted = false;           // already in (col, row) order
};

namespace {

bsp_status fail(bsp_status st, const std::string &msg) {
  bsp::set_error(msg);
  return st;
}

int nthreads(int32_t t) { return t > 0 ? t : std::max(1, omp_get_max_threads()); }

inline bool blank(char ch) { return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\v' || ch == '\f'; }

inline const char *eol(const char *p, const char *e) {
  const void *q = memchr(p, '\n', (size_t)(e - p));
  return q ? static_cast<const char *>(q) : e;
}

inline const char *skip_blank(const char *p, const char *e) {
  while (p < e && blank(*p)) ++p;
  return p;
}

struct Mapped {
  const char *p = nullptr;
  size_t n = 0;
  int fd = -1;
  ~Mapped() {
    if (p) munmap(const_cast<char *>(p), n);
    if (fd >= 0) close(fd);
  }
};

bsp_status map_file(const char *path, Mapped &m) {
  m.fd = open(path, O_RDONLY);
  if (m.fd < 0) return fail(BSP_ERR_INVALID, std::string("cannot open ") + path);
  struct stat st;
  if (fstat(m.fd, &st) != 0) return fail(BSP_ERR_INVALID, std::string("cannot stat ") + path);
  m.n = (size_t)st.st_size;
  if (m.n == 0) return fail(BSP_ERR_INVALID, std::string("empty file ") + path);
  void *q = mmap(nullptr, m.n, PROT_READ, MAP_PRIVATE, m.fd, 0);
  if (q == MAP_FAILED) return fail(BSP_ERR_INVALID, std::string("cannot map ") + path);
  m.p = static_cast<const char *>(q);
  madvise(q, m.n, MADV_SEQUENTIAL);
  return BSP_OK;
}

std::vector<std::string> tokens(const char *p, const char *e) {
  std::vector<std::string> t;
  while (true) {
    p = skip_blank(p, e);
    if (p >= e) break;
    const char *q = p;
    while (q < e && !blank(*q)) ++q;
    std::string s(p, q);
    for (char &ch : s) ch = (char)tolower((unsigned char)ch);
    t.push_back(s);
    p = q;
  }
  return t;
}

inline bool parse_i64(const char *&p, const char *e, int64_t &out) {
  p = skip_blank(p, e);
  const auto r = std::from_chars(p, e, out);
  if (r.ec != std::errc()) return false;
  p = r.ptr;
  return true;
}

inline bool parse_f64(const char *&p, const char *e, double &out) {
  p = skip_blank(p, e);
  const auto r = std::from_chars(p, e, out);  // no leading '+', as fast_float
  // out of range: from_chars leaves `out` untouched; give the IEEE result
  if (r.ec == std::errc::result_out_of_range) {
    out = strtod(std::string(p, r.ptr).c_str(), nullptr);
  } else if (r.ec != std::errc()) {
    return false;
  }
  p = r.ptr;
  return true;
}

struct Header {
  int format = BSP_MTX_COORDINATE, field = BSP_MTX_REAL, symmetry = BSP_MTX_GENERAL;
  int64_t rows = 0, cols = 0, entries = 0;
  const char *body = nullptr;
};

bsp_status parse_header(const char *b, const char *e, Header &h) {
  const char *le = eol(b, e);
  const auto t = tokens(b, le);
  // the banner word is case-sensitive (fast_matrix_market rejects other
  // spellings); the words after it are not
  if (t.empty() || t[0] != "%%matrixmarket" || strncmp(b, "%%MatrixMarket", 14) != 0)
    return fail(BSP_ERR_INVALID, "missing %%MatrixMarket banner");
  if (t.size() < 5) return fail(BSP_ERR_INVALID, "banner needs object, format, field and symmetry");
  if (t[1] != "matrix") return fail(BSP_ERR_UNSUPPORTED, "object '" + t[1] + "' (only 'matrix')");
  if (t[2] == "coordinate")
    h.format = BSP_MTX_COORDINATE;
  else if (t[2] == "array")
    h.format = BSP_MTX_ARRAY;
  else
    return fail(BSP_ERR_INVALID, "format '" + t[2] + "'");
  if (t[3] == "real" || t[3] == "double")
    h.field = BSP_MTX_REAL;
  else if (t[3] == "integer")
    h.field = BSP_MTX_INTEGER;
  else if (t[3] == "pattern")
    h.field = BSP_MTX_PATTERN;
  else if (t[3] == "complex")
    return fail(BSP_ERR_UNSUPPORTED, "complex values");
  else
    return fail(BSP_ERR_INVALID, "field '" + t[3] + "'");
  if (t[4] == "general")
    h.symmetry = BSP_MTX_GENERAL;
  else if (t[4] == "symmetric")
    h.symmetry = BSP_MTX_SYMMETRIC;
  else if (t[4] == "skew-symmetric")
    h.symmetry = BSP_MTX_SKEW_SYMMETRIC;
  else if (t[4] == "hermitian")
    h.symmetry = BSP_MTX_HERMITIAN;
  else
    return fail(BSP_ERR_INVALID, "symmetry '" + t[4] + "'");
  if (h.format == BSP_MTX_ARRAY && h.field == BSP_MTX_PATTERN)
    return fail(BSP_ERR_INVALID, "an array file cannot be 'pattern'");
  const char *p = le < e ? le + 1 : e;
  while (p < e) {
    const char *l = eol(p, e);
    const char *q = skip_blank(p, l);
    if (q == l || *q == '%') {
      p = l < e ? l + 1 : e;
      continue;
    }
    const char *s = q;
    int64_t v[3] = {0, 0, 0};
    const int need = h.format == BSP_MTX_COORDINATE ? 3 : 2;
    for (int k = 0; k < need; ++k)
      if (!parse_i64(s, l, v[k]) || v[k] < 0) return fail(BSP_ERR_INVALID, "malformed size line");
    h.rows = v[0];
    h.cols = v[1];
    h.entries = need == 3 ? v[2] : 0;
    h.body = l < e ? l + 1 : e;
    return BSP_OK;
  }
  return fail(BSP_ERR_INVALID, "missing size line");
}

// Byte ranges of [b, e) for T threads, each starting at a line start.
std::vector<const char *> split(const char *b, const char *e, int T) {
  std::vector<const char *> cut(T + 1, e);
  cut[0] = b;
  const size_t n = (size_t)(e - b);
  for (int t = 1; t < T; ++t) {
    const char *p = b + n * (size_t)t / (size_t)T;
    p = std::max(p, cut[t - 1]);
    if (p > b && p < e && p[-1] != '\n') p = std::min(e, eol(p, e) + 1);
    cut[t] = p;
  }
  return cut;
}

// Data lines in [b, e): not blank and not starting with '%'.
int64_t count_lines(const char *b, const char *e) {
  int64_t n = 0;
  const char *p = b;
  while (p < e) {
    const char *l = eol(p, e);
    const char *q = skip_blank(p, l);
    n += (q < l && *q != '%');
    p = l < e ? l + 1 : e;
  }
  return n;
}

struct Part {
  int64_t off = 0, count = 0, offdiag = 0;
  bool row_sorted = true;  // (row, col) non-decreasing inside the range
  bool col_sorted = true;  // (col, row) non-decreasing inside the range
  bsp_status st = BSP_OK;
  std::string msg;
};

// One thread's lines, written straight into the triplet arrays at P.off.
void parse_range(const char *b, const char *e, const Header &h, Part &P, int32_t *R, int32_t *Cc, double *V) {
  const bool coord = h.format == BSP_MTX_COORDINATE, pattern = h.field == BSP_MTX_PATTERN;
  int64_t k = P.off;
  const int64_t end = P.off + P.count;
  uint64_t prev = 0, prev2 = 0;
  const char *p = b;
  while (p < e && k < end) {
    const char *l = eol(p, e);
    const char *q = skip_blank(p, l);
    const char *next = l < e ? l + 1 : e;
    if (q == l || *q == '%') {
      p = next;
      continue;
    }
    if (coord) {
      int64_t i, j;
      if (!parse_i64(q, l, i) || !parse_i64(q, l, j)) {
        P.st = BSP_ERR_INVALID;
        P.msg = "malformed entry: '" + std::string(p, std::min<size_t>(l - p, 80)) + "'";
        return;
      }
      if (i < 1 || i > h.rows || j < 1 || j > h.cols) {
        P.st = BSP_ERR_INVALID;
        P.msg = "index out of range: '" + std::string(p, std::min<size_t>(l - p, 80)) + "'";
        return;
      }
      R[k] = (int32_t)(i - 1);
      Cc[k] = (int32_t)(j - 1);
      P.offdiag += i != j;
      const uint64_t key = ((uint64_t)(i - 1) << 32) | (uint64_t)(j - 1);
      const uint64_t key2 = ((uint64_t)(j - 1) << 32) | (uint64_t)(i - 1);
      if (k > P.off && key < prev) P.row_sorted = false;
      if (k > P.off && key2 < prev2) P.col_sorted = false;
      prev = key;
      prev2 = key2;
    }
    if (pattern) {
      V[k] = 1.0;
    } else if (!parse_f64(q, l, V[k])) {
      P.st = BSP_ERR_INVALID;
      P.msg = "malformed value: '" + std::string(p, std::min<size_t>(l - p, 80)) + "'";
      return;
    }
    ++k;
    p = next;
  }
}

bsp_status read_body(const char *b, const char *e, const Header &h, int T, int32_t flags, bsp_mtx_s &M) {
  const bool coord = h.format == BSP_MTX_COORDINATE;
  const bool general = h.symmetry == BSP_MTX_GENERAL;
  const bool skew = h.symmetry == BSP_MTX_SKEW_SYMMETRIC;
  if (h.rows > INT32_MAX || h.cols > INT32_MAX) return fail(BSP_ERR_UNSUPPORTED, "dimensions above 2^31-1");
  if (!general && h.rows != h.cols) return fail(BSP_ERR_INVALID, "a symmetric file must be square");
  int64_t expect = h.entries;
  if (!coord) {
    const int64_t n = h.rows;
    if (general && h.rows > 0 && h.cols > INT32_MAX / h.rows) return fail(BSP_ERR_UNSUPPORTED, "array too large");
    expect = general ? h.rows * h.cols : (skew ? n * (n - 1) / 2 : n * (n + 1) / 2);
  }
  if (expect > INT32_MAX) return fail(BSP_ERR_UNSUPPORTED, "more than 2^31-1 entries");
  const size_t bytes = (size_t)(e - b);
  T = (int)std::max<size_t>(1, std::min<size_t>((size_t)T, bytes / (1 << 16) + 1));
  const auto cut = split(b, e, T);
  // pass 1: data lines per range -> where each range writes
  std::vector<Part> part(T);
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t) part[t].count = count_lines(cut[t], cut[t + 1]);
  int64_t got = 0;
  for (int t = 0; t < T; ++t) {
    part[t].off = got;
    got += part[t].count;
  }
  if (got != expect)
    return fail(BSP_ERR_INVALID, "the file holds " + std::to_string(got) + " entries, its size line says " +
                                     std::to_string(expect));
  // room for the mirrors too; pages are first touched by the writing threads
  const int64_t cap = general ? got : 2 * got;
  if (cap > 0) {
    M.r.reset(new int32_t[cap]);
    M.c.reset(new int32_t[cap]);
    M.v.reset(new double[cap]);
  }
  int32_t *R = M.r.get(), *Cc = M.c.get();
  double *V = M.v.get();
  // pass 2: parse
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t) parse_range(cut[t], cut[t + 1], h, part[t], R, Cc, V);
  for (int t = 0; t < T; ++t)
    if (part[t].st != BSP_OK) return fail(part[t].st, part[t].msg);
  // global order = every range in order and every seam in order
  bool sorted = coord, csorted = coord;
  const auto rkey = [&](int64_t k) { return (uint64_t)(uint32_t)R[k] << 32 | (uint32_t)Cc[k]; };
  const auto ckey = [&](int64_t k) { return (uint64_t)(uint32_t)Cc[k] << 32 | (uint32_t)R[k]; };
  for (int t = 0; t < T; ++t) {
    sorted = sorted && part[t].row_sorted;
    csorted = csorted && part[t].col_sorted;
    if (part[t].count && part[t].off > 0) {
      const int64_t k = part[t].off;
      sorted = sorted && rkey(k - 1) <= rkey(k);
      csorted = csorted && ckey(k - 1) <= ckey(k);
    }
  }
  if (!coord) {
    const int64_t n = h.rows;
    if (general) {
#pragma omp parallel for num_threads(T) schedule(static)
      for (int64_t k = 0; k < got; ++k) {
        R[k] = (int32_t)(k % n);
        Cc[k] = (int32_t)(k / n);
      }
    } else {
      // column j holds rows j..n-1 (j+1..n-1 for skew), column-major
#pragma omp parallel for num_threads(T) schedule(dynamic, 64)
      for (int64_t j = 0; j < n; ++j) {
        const int64_t first = skew ? j + 1 : j;
        const int64_t start = skew ? j * (n - 1) - j * (j - 1) / 2 : j * n - j * (j - 1) / 2;
        for (int64_t i = first; i < n; ++i) {
          R[start + i - first] = (int32_t)i;
          Cc[start + i - first] = (int32_t)j;
        }
      }
    }
    // array files are column-major: (col, row) order when general
    sorted = general && h.cols <= 1;
    csorted = general;
  }
  // symmetry expansion: mirrors after the stored entries, in file order
  const bool expand = !general && !(flags & BSP_MTX_NO_EXPAND);
  const bool diag_zero = expand && (flags & BSP_MTX_DIAG_ZERO);
  const bool diag_dup = expand && (flags & BSP_MTX_DIAG_DUPLICATE);
  const bool diag_copy = diag_zero || diag_dup;
  std::vector<int64_t> moff(T + 1, 0);
  const auto tcut = [&](int t) { return got * t / T; };
  if (expand) {
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
      int64_t m = 0;
      for (int64_t k = tcut(t); k < tcut(t + 1); ++k) m += (R[k] != Cc[k]) || diag_copy;
      moff[t + 1] = m;
    }
    for (int t = 0; t < T; ++t) moff[t + 1] += moff[t];
  }
  const int64_t nnz = got + moff[T];
  if (nnz > INT32_MAX) return fail(BSP_ERR_UNSUPPORTED, "more than 2^31-1 entries after the symmetry expansion");
  if (expand) {
    const double sign = skew ? -1.0 : 1.0;
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
      int64_t o = got + moff[t];
      for (int64_t k = tcut(t); k < tcut(t + 1); ++k) {
        if (R[k] != Cc[k]) {
          R[o] = Cc[k];
          Cc[o] = R[k];
          V[o] = sign * V[k];
          ++o;
        } else if (diag_copy) {
          R[o] = R[k];
          Cc[o] = Cc[k];
          V[o] = diag_zero ? 0.0 : V[k];
          ++o;
        }
      }
    }
    if (nnz > got) sorted = csorted = false;
  }
  M.info.rows = h.rows;
  M.info.cols = h.cols;
  M.info.entries = got;
  M.info.nnz = nnz;
  M.info.format = h.format;
  M.info.field = h.field;
  M.info.symmetry = h.symmetry;
  M.sorted = sorted;
  M.col_sorted = csorted;
  return BSP_OK;
}

}  // namespace

static bsp_status read_text(const char *p, size_t n, int32_t flags, int32_t threads, bsp_mtx *out) {
  if (flags & ~(BSP_MTX_DIAG_ZERO | BSP_MTX_DIAG_DUPLICATE | BSP_MTX_NO_EXPAND))
    return fail(BSP_ERR_INVALID, "bsp_mtx_read: unknown flags");
  if ((flags & BSP_MTX_DIAG_ZERO) && (flags & BSP_MTX_DIAG_DUPLICATE))
    return fail(BSP_ERR_INVALID, "bsp_mtx_read: DIAG_ZERO and DIAG_DUPLICATE exclude each other");
  Header h;
  bsp_status st = parse_header(p, p + n, h);
  if (st != BSP_OK) return st;
  auto *M = new (std::nothrow) bsp_mtx_s();
  if (!M) return fail(BSP_ERR_ALLOC, "bsp_mtx_read: out of host memory");
  try {
    st = read_body(h.body, p + n, h, nthreads(threads), flags, *M);
  } catch (const std::bad_alloc &) {
    st = fail(BSP_ERR_ALLOC, "bsp_mtx_read: out of host memory");
  }
  if (st != BSP_OK) {
    delete M;
    return st;
  }
  *out = M;
  return BSP_OK;
}

extern "C" bsp_status bsp_mtx_read(const char *path, int32_t flags, int32_t threads, bsp_mtx *out) {
  bsp::clear_error();
  if (!path || !out) return fail(BSP_ERR_INVALID, "bsp_mtx_read: null pointer");
  *out = nullptr;
  Mapped f;
  const bsp_status st = map_file(path, f);
  if (st != BSP_OK) return st;
  return read_text(f.p, f.n, flags, threads, out);
}

extern "C" bsp_status bsp_mtx_read_buffer(const char *data, size_t bytes, int32_t flags, int32_t threads,
                                          bsp_mtx *out) {
  bsp::clear_error();
  if (!data || !out) return fail(BSP_ERR_INVALID, "bsp_mtx_read_buffer: null pointer");
  *out = nullptr;
  if (bytes == 0) return fail(BSP_ERR_INVALID, "bsp_mtx_read_buffer: empty buffer");
  return read_text(data, bytes, flags, threads, out);
}

extern "C" bsp_status bsp_mtx_get_info(bsp_mtx m, bsp_mtx_info *info) {
  bsp::clear_error();
  if (!m || !info) return fail(BSP_ERR_INVALID, "bsp_mtx_get_info: null pointer");
  *info = m->info;
  return BSP_OK;
}

extern "C" bsp_status bsp_mtx_triplets(bsp_mtx m, int32_t *rows, int32_t *cols, double *values) {
  bsp::clear_error();
  if (!m) return fail(BSP_ERR_INVALID, "bsp_mtx_triplets: null handle");
  const int64_t n = m->info.nnz;
  if (rows) std::copy(m->r.get(), m->r.get() + n, rows);
  if (cols) std::copy(m->c.get(), m->c.get() + n, cols);
  if (values) std::copy(m->v.get(), m->v.get() + n, values);
  return BSP_OK;
}

extern "C" bsp_status bsp_mtx_csr_host(bsp_mtx m, int32_t *rowPtr, int32_t *colIdx, double *values) {
  bsp::clear_error();
  if (!m || !rowPtr || (m->info.nnz && (!colIdx || !values)))
    return fail(BSP_ERR_INVALID, "bsp_mtx_csr_host: null pointer");
  const int64_t n = m->info.nnz;
  const int32_t rows = (int32_t)m->info.rows;
  const int T = nthreads(0);
  try {
    std::vector<int32_t> cnt((size_t)rows + 1, 0);
    const int32_t *R = m->r.get(), *Cc = m->c.get();
    const double *Vv = m->v.get();
    if (m->sorted) {  // already in CSR order: count rows, copy
#pragma omp parallel for num_threads(T) schedule(static)
      for (int64_t k = 0; k < n; ++k) __atomic_fetch_add(&cnt[R[k] + 1], 1, __ATOMIC_RELAXED);
      rowPtr[0] = 0;
      for (int32_t i = 0; i < rows; ++i) rowPtr[i + 1] = rowPtr[i] + cnt[i + 1];
#pragma omp parallel for num_threads(T) schedule(static)
      for (int64_t k = 0; k < n; ++k) {
        colIdx[k] = Cc[k];
        values[k] = Vv[k];
      }
      return BSP_OK;
    }
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t k = 0; k < n; ++k) __atomic_fetch_add(&cnt[R[k] + 1], 1, __ATOMIC_RELAXED);
    rowPtr[0] = 0;
    for (int32_t i = 0; i < rows; ++i) rowPtr[i + 1] = rowPtr[i] + cnt[i + 1];
    std::vector<int32_t> cur(rowPtr, rowPtr + rows);
    std::vector<uint64_t> key((size_t)n);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int64_t k = 0; k < n; ++k) {
      const int32_t pos = __atomic_fetch_add(&cur[R[k]], 1, __ATOMIC_RELAXED);
      key[pos] = ((uint64_t)(uint32_t)Cc[k] << 32) | (uint64_t)(uint32_t)k;
    }
#pragma omp parallel for num_threads(T) schedule(dynamic, 2048)
    for (int32_t i = 0; i < rows; ++i) {
      uint64_t *a = key.data() + rowPtr[i];
      const int32_t len = rowPtr[i + 1] - rowPtr[i];
      if (len <= 32) {
        for (int32_t x = 1; x < len; ++x) {
          const uint64_t t = a[x];
          int32_t y = x - 1;
          while (y >= 0 && a[y] > t) {
            a[y + 1] = a[y];
            --y;
          }
          a[y + 1] = t;
        }
      } else {
        std::sort(a, a + len);
      }
      for (int32_t x = 0; x < len; ++x) {
        colIdx[rowPtr[i] + x] = (int32_t)(a[x] >> 32);
        values[rowPtr[i] + x] = Vv[(size_t)(uint32_t)a[x]];
      }
    }
  } catch (const std::bad_alloc &) {
    return fail(BSP_ERR_ALLOC, "bsp_mtx_csr_host: out of host memory");
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_mtx_csr(bsp_mtx m, int32_t *rowPtr, int32_t *colIdx, double *values,
                                  bsp_stream_t stream) {
  bsp::clear_error();
  if (!m || !rowPtr || (m->info.nnz && (!colIdx || !values)))
    return fail(BSP_ERR_INVALID, "bsp_mtx_csr: null pointer");
  return bsp::mtx_csr_device((int32_t)m->info.rows, (int32_t)m->info.cols, m->info.nnz, m->r.get(), m->c.get(),
                             m->v.get(), m->sorted, m->col_sorted, rowPtr, colIdx, values,
                             reinterpret_cast<cudaStream_t>(stream));
}

extern "C" bsp_status bsp_mtx_free(bsp_mtx m) {
  bsp::clear_error();
  delete m;
  return BSP_OK;
}

extern "C" bsp_status bsp_mtx_write_csr_host(const char *path, int32_t rows, int32_t cols, int64_t nnz,
                                             const int32_t *rowPtr, const int32_t *colIdx, const double *values,
                                             int32_t threads) {
  bsp::clear_error();
  if (!path || !rowPtr || (nnz && !colIdx) || rows < 0 || cols < 0 || nnz < 0)
    return fail(BSP_ERR_INVALID, "bsp_mtx_write_csr_host: bad argument");
  if (rowPtr[0] != 0 || rowPtr[rows] != nnz) return fail(BSP_ERR_INVALID, "bsp_mtx_write_csr_host: bad rowPtr");
  FILE *f = fopen(path, "wb");
  if (!f) return fail(BSP_ERR_INVALID, std::string("cannot create ") + path);
  const int T = nthreads(threads);
  std::string head = std::string("%%MatrixMarket matrix coordinate ") + (values ? "real" : "pattern") +
                     " general\n" + std::to_string(rows) + " " + std::to_string(cols) + " " + std::to_string(nnz) +
                     "\n";
  bool ok = fwrite(head.data(), 1, head.size(), f) == head.size();
  // rounds of T row ranges holding about 4M entries each
  const int64_t per = 1 << 22;
  int32_t r0 = 0;
  std::vector<std::string> buf(T);
  while (ok && r0 < rows) {
    std::vector<int32_t> cut(T + 1, r0);
    for (int t = 1; t <= T; ++t) {
      const int64_t target = rowPtr[cut[t - 1]] + per;
      cut[t] = (int32_t)(std::upper_bound(rowPtr + cut[t - 1], rowPtr + rows + 1, (int32_t)std::min<int64_t>(
                                              target, INT32_MAX)) - rowPtr - 1);
      cut[t] = std::max(cut[t], std::min(rows, cut[t - 1] + 1));
    }
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
      std::string &s = buf[t];
      s.clear();
      char tmp[64];
      for (int32_t i = cut[t]; i < cut[t + 1]; ++i)
        for (int32_t k = rowPtr[i]; k < rowPtr[i + 1]; ++k) {
          char *p = tmp;
          p = std::to_chars(p, tmp + sizeof tmp, (int64_t)i + 1).ptr;
          *p++ = ' ';
          p = std::to_chars(p, tmp + sizeof tmp, (int64_t)colIdx[k] + 1).ptr;
          if (values) {
            *p++ = ' ';
            p = std::to_chars(p, tmp + sizeof tmp, values[k]).ptr;
          }
          *p++ = '\n';
          s.append(tmp, p);
        }
    }
    for (int t = 0; t < T && ok; ++t) ok = fwrite(buf[t].data(), 1, buf[t].size(), f) == buf[t].size();
    r0 = cut[T];
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) return fail(BSP_ERR_INVALID, std::string("write failed: ") + path);
  return BSP_OK;
}
