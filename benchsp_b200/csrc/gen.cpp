// Seeded synthetic matrix generators (host, OpenMP).  They stand in for the
// SuiteSparse .mtx inputs the reference's bench drivers read
// (bench/spmvfp64.cpp:37-42); the banded power-law shape follows the
// reference's own generator (gendata.cpp:5-13, n = 2^21).
//
// Every random draw is a counter-based hash of (seed, stream, index), so the
// output does not depend on the thread count and the count pass and the fill
// pass see identical matrices.  All generators emit CSR with ascending,
// distinct column indices.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/bsp.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t h3(uint64_t seed, uint64_t a, uint64_t b) {
  return mix64(mix64(mix64(seed) ^ a) ^ (b * 0xD6E8FEB86659FD93ull));
}
// Uniform in (0, 1): 53 random bits, never 0.
inline double u01(uint64_t h) { return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
inline double normal(uint64_t seed, uint64_t stream, uint64_t idx) {
  const double u1 = u01(h3(seed, stream, 2 * idx));
  const double u2 = u01(h3(seed, stream, 2 * idx + 1));
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// Exclusive prefix of per-row counts into rowPtr (serial; rows <= 2^31).
inline int64_t prefix(const std::vector<int32_t> &cnt, int32_t *rowPtr) {
  int64_t acc = 0;
  for (size_t i = 0; i < cnt.size(); ++i) {
    if (rowPtr) rowPtr[i] = (int32_t)acc;
    acc += cnt[i];
  }
  if (rowPtr) rowPtr[cnt.size()] = (int32_t)acc;
  return acc;
}

enum : uint64_t { kStreamVal = 1, kStreamLen = 2, kStreamCol = 3, kStreamFill = 4, kStreamMask = 5, kStreamX = 6 };

}  // namespace

extern "C" bsp_status bsp_gen_laplace2d(int32_t nx, int32_t ny, int32_t *rows, int32_t *nnz, int32_t *rowPtr,
                                        int32_t *colIdx, double *values) {
  if (nx <= 0 || ny <= 0 || !rows || !nnz) return BSP_ERR_INVALID;
  const int64_t n = (int64_t)nx * ny;
  const int64_t z = 5 * n - 2 * (int64_t)nx - 2 * (int64_t)ny;
  if (n > INT32_MAX || z > INT32_MAX) return BSP_ERR_INVALID;
  *rows = (int32_t)n;
  *nnz = (int32_t)z;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % nx, y = i / nx;
    // Row start in closed form: 5 per earlier row minus the neighbours that
    // earlier rows miss at the four grid edges.
    const int64_t before_south = std::min<int64_t>(i, nx);          // rows with y==0 before i
    const int64_t before_north = std::max<int64_t>(0, i - (n - nx));  // rows with y==ny-1 before i
    const int64_t before_west = y + (x > 0 ? 1 : 0);                 // rows with x==0 before i
    const int64_t before_east = y;                                   // rows with x==nx-1 before i
    const int64_t start = 5 * i - before_south - before_north - before_west - before_east;
    rowPtr[i] = (int32_t)start;
    int64_t k = start;
    auto put = [&](int64_t c, double v) {
      colIdx[k] = (int32_t)c;
      values[k] = v;
      ++k;
    };
    if (y > 0) put(i - nx, -1.0);
    if (x > 0) put(i - 1, -1.0);
    put(i, 4.0);
    if (x < nx - 1) put(i + 1, -1.0);
    if (y < ny - 1) put(i + nx, -1.0);
  }
  rowPtr[n] = (int32_t)z;
  return BSP_OK;
}

extern "C" bsp_status bsp_gen_poisson3d(int32_t m, int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                                        int32_t *colIdx, double *values) {
  if (m <= 0 || !rows || !nnz) return BSP_ERR_INVALID;
  const int64_t n = (int64_t)m * m * m;
  if (n > INT32_MAX) return BSP_ERR_INVALID;
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % m, y = (i / m) % m, z = i / ((int64_t)m * m);
    cnt[i] = 1 + (x > 0) + (x < m - 1) + (y > 0) + (y < m - 1) + (z > 0) + (z < m - 1);
  }
  *rows = (int32_t)n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (!rowPtr) return BSP_OK;
  const int64_t m2 = (int64_t)m * m;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % m, y = (i / m) % m, z = i / m2;
    int64_t k = rowPtr[i];
    auto put = [&](int64_t c, double v) {
      colIdx[k] = (int32_t)c;
      values[k] = v;
      ++k;
    };
    if (z > 0) put(i - m2, -1.0);
    if (y > 0) put(i - m, -1.0);
    if (x > 0) put(i - 1, -1.0);
    put(i, 6.0);
    if (x < m - 1) put(i + 1, -1.0);
    if (y < m - 1) put(i + m, -1.0);
    if (z < m - 1) put(i + m2, -1.0);
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_gen_stencil27(int32_t m, int32_t dof, uint64_t seed, int32_t *rows, int64_t *nnz,
                                        int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (m <= 0 || dof <= 0 || !rows || !nnz) return BSP_ERR_INVALID;
  const int64_t nodes = (int64_t)m * m * m;
  const int64_t n = nodes * dof;
  if (n > INT32_MAX) return BSP_ERR_INVALID;
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t node = 0; node < nodes; ++node) {
    const int64_t x = node % m, y = (node / m) % m, z = node / ((int64_t)m * m);
    const int nb = (1 + (x > 0) + (x < m - 1)) * (1 + (y > 0) + (y < m - 1)) * (1 + (z > 0) + (z < m - 1));
    for (int d = 0; d < dof; ++d) cnt[node * dof + d] = nb * dof;
  }
  *rows = (int32_t)n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (total > INT32_MAX) return BSP_ERR_INVALID;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel for schedule(static)
  for (int64_t node = 0; node < nodes; ++node) {
    const int64_t x = node % m, y = (node / m) % m, z = node / ((int64_t)m * m);
    for (int d = 0; d < dof; ++d) {
      const int64_t row = node * dof + d;
      int64_t k = rowPtr[row];
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int64_t xx = x + dx, yy = y + dy, zz = z + dz;
            if (xx < 0 || yy < 0 || zz < 0 || xx >= m || yy >= m || zz >= m) continue;
            const int64_t nbr = (zz * m + yy) * m + xx;
            for (int e = 0; e < dof; ++e) {
              colIdx[k] = (int32_t)(nbr * dof + e);
              values[k] = normal(seed, kStreamVal, (uint64_t)k);
              ++k;
            }
          }
    }
  }
  return BSP_OK;
}

namespace {
// Distinct sorted draws of `count` values from [0, range) for stream `row`.
void distinct_draws(uint64_t seed, uint64_t stream, uint64_t row, int64_t count, int64_t range,
                    std::vector<int32_t> &out) {
  out.clear();
  if (count >= range) {
    for (int64_t c = 0; c < range; ++c) out.push_back((int32_t)c);
    return;
  }
  uint64_t draw = 0;
  while ((int64_t)out.size() < count) {
    while ((int64_t)out.size() < count)
      out.push_back((int32_t)(h3(seed, stream, (row << 24) ^ draw++) % (uint64_t)range));
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  }
}

struct BlockMask {
  uint64_t w[4] = {0, 0, 0, 0};
  bool get(int e) const { return (w[e >> 6] >> (e & 63)) & 1; }
  void set(int e) { w[e >> 6] |= 1ull << (e & 63); }
  bool empty() const { return !(w[0] | w[1] | w[2] | w[3]); }
};

BlockMask block_mask(uint64_t seed, int64_t br, int k, int bs, double lo, double hi) {
  const int ne = bs * bs;
  const double p = lo + (hi - lo) * u01(h3(seed, kStreamFill, ((uint64_t)br << 8) | (uint64_t)k));
  BlockMask m;
  for (int e = 0; e < ne; ++e) {
    const uint64_t idx = bs <= 8 ? (((uint64_t)br << 14) | ((uint64_t)k << 7) | (uint64_t)e)
                                 : (((uint64_t)br << 16) | ((uint64_t)k << 8) | (uint64_t)e);
    if (u01(h3(seed, kStreamMask, idx)) < p) m.set(e);
  }
  if (m.empty()) m.set((int)(h3(seed, kStreamMask, ~(uint64_t)br ^ (uint64_t)k) % ne));
  return m;
}
}  // namespace

extern "C" bsp_status bsp_gen_random_bsr(int32_t nbr, int32_t bs, int32_t per_row, double fill_lo,
                                         double fill_hi, uint64_t seed, int32_t *rows, int64_t *nnz,
                                         int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (nbr <= 0 || (bs != 4 && bs != 8 && bs != 16) || per_row <= 0 || per_row > 255 || !rows || !nnz)
    return BSP_ERR_INVALID;
  const int64_t n = (int64_t)nbr * bs;
  if (n > INT32_MAX) return BSP_ERR_INVALID;
  std::vector<int32_t> cnt(n, 0);
#pragma omp parallel
  {
    std::vector<int32_t> bc;
#pragma omp for schedule(static)
    for (int64_t br = 0; br < nbr; ++br) {
      distinct_draws(seed, kStreamCol, (uint64_t)br, per_row, nbr, bc);
      for (int k = 0; k < (int)bc.size(); ++k) {
        const BlockMask mask = block_mask(seed, br, k, bs, fill_lo, fill_hi);
        for (int i = 0; i < bs; ++i)
          for (int j = 0; j < bs; ++j) cnt[br * bs + i] += mask.get(i * bs + j);
      }
    }
  }
  *rows = (int32_t)n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (total > INT32_MAX) return BSP_ERR_INVALID;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel
  {
    std::vector<int32_t> bc;
    std::vector<BlockMask> masks;
#pragma omp for schedule(static)
    for (int64_t br = 0; br < nbr; ++br) {
      distinct_draws(seed, kStreamCol, (uint64_t)br, per_row, nbr, bc);
      masks.resize(bc.size());
      for (int k = 0; k < (int)bc.size(); ++k) masks[k] = block_mask(seed, br, k, bs, fill_lo, fill_hi);
      for (int i = 0; i < bs; ++i) {
        const int64_t row = br * bs + i;
        int64_t kk = rowPtr[row];
        for (int k = 0; k < (int)bc.size(); ++k)
          for (int j = 0; j < bs; ++j)
            if (masks[k].get(i * bs + j)) {
              colIdx[kk] = (int32_t)((int64_t)bc[k] * bs + j);
              values[kk] = normal(seed, kStreamVal, (uint64_t)kk);
              ++kk;
            }
      }
    }
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_gen_powerlaw(int32_t n, double alpha, int32_t max_len, uint64_t seed, int32_t *rows,
                                       int64_t *nnz, int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (n <= 0 || max_len <= 0 || alpha <= 0.0 || !rows || !nnz) return BSP_ERR_INVALID;
  if (max_len > n) max_len = n;
  // Inverse-CDF table of Zipf(alpha) on [1, max_len].
  std::vector<double> cdf(max_len);
  double acc = 0.0;
  for (int32_t k = 1; k <= max_len; ++k) {
    acc += pow((double)k, -alpha);
    cdf[k - 1] = acc;
  }
  for (auto &c : cdf) c /= acc;
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double u = u01(h3(seed, kStreamLen, (uint64_t)i));
    cnt[i] = (int32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
  }
  *rows = n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (total > INT32_MAX) return BSP_ERR_INVALID;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel
  {
    std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
      distinct_draws(seed, kStreamCol, (uint64_t)i, cnt[i], n, cols);
      int64_t k = rowPtr[i];
      for (int32_t c : cols) {
        colIdx[k] = c;
        values[k] = normal(seed, kStreamVal, (uint64_t)k);
        ++k;
      }
    }
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_gen_uniform(int64_t n, uint64_t seed, double *x) {
  if (n < 0 || (n > 0 && !x)) return BSP_ERR_INVALID;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = 2.0 * u01(h3(seed, kStreamX, (uint64_t)i)) - 1.0;
  return BSP_OK;
}

// Power-law graph for the SpMM benchmark: out-degrees ~ Zipf(alpha) on
// [1, d_max] with d_max chosen so the mean degree is `mean_deg` (bisection),
// distinct uniform targets, values 1/degree (row-stochastic).
extern "C" bsp_status bsp_gen_graph(int32_t n, double alpha, double mean_deg, uint64_t seed, int32_t *rows,
                                    int64_t *nnz, int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (n <= 0 || alpha <= 1.0 || mean_deg < 1.0 || !rows || !nnz) return BSP_ERR_INVALID;
  // prefix sums of k^-alpha and k^(1-alpha): mean(dmax) = S1[dmax] / S0[dmax]
  std::vector<double> S0(n + 1, 0.0), S1(n + 1, 0.0);
  for (int64_t k = 1; k <= n; ++k) {
    const double p = pow((double)k, -alpha);
    S0[k] = S0[k - 1] + p;
    S1[k] = S1[k - 1] + p * (double)k;
  }
  auto mean_for = [&](int64_t dmax) { return S1[dmax] / S0[dmax]; };
  int64_t lo = 1, hi = n;
  if (mean_for(hi) < mean_deg) return BSP_ERR_INVALID;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) / 2;
    (mean_for(mid) < mean_deg ? lo : hi) = mid;
  }
  const int64_t dmax = hi;
  std::vector<double> cdf(dmax);
  double acc = 0.0;
  for (int64_t k = 1; k <= dmax; ++k) {
    acc += pow((double)k, -alpha);
    cdf[k - 1] = acc;
  }
  for (auto &c : cdf) c /= acc;
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double u = u01(h3(seed, kStreamLen, (uint64_t)i));
    cnt[i] = (int32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
  }
  *rows = n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (total > INT32_MAX) return BSP_ERR_INVALID;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel
  {
    std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; ++i) {
      distinct_draws(seed, kStreamCol, (uint64_t)i, cnt[i], n, cols);
      int64_t k = rowPtr[i];
      for (int32_t c : cols) {
        colIdx[k] = c;
        values[k] = 1.0 / (double)cnt[i];
        ++k;
      }
    }
  }
  return BSP_OK;
}

// Banded matrix: row i holds columns [i - (width-1)/2, i + width/2] clipped to
// [0, n), values N(0, 1).
extern "C" bsp_status bsp_gen_banded(int32_t n, int32_t width, uint64_t seed, int32_t *rows, int64_t *nnz,
                                     int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (n <= 0 || width <= 0 || !rows || !nnz) return BSP_ERR_INVALID;
  const int32_t lo = (width - 1) / 2, hi = width / 2;
  std::vector<int32_t> cnt(n);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t a = std::max<int64_t>(0, i - lo), b = std::min<int64_t>(n - 1, i + hi);
    cnt[i] = (int32_t)(b - a + 1);
  }
  *rows = n;
  const int64_t total = prefix(cnt, rowPtr);
  *nnz = total;
  if (total > INT32_MAX) return BSP_ERR_INVALID;
  if (!rowPtr) return BSP_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t k = rowPtr[i];
    for (int64_t c = std::max<int64_t>(0, i - lo); c <= std::min<int64_t>(n - 1, i + hi); ++c, ++k) {
      colIdx[k] = (int32_t)c;
      values[k] = normal(seed, kStreamVal, (uint64_t)k);
    }
  }
  return BSP_OK;
}

// ---------------------------------------------------------------------------
// SPD test matrices for preconditioned CG.
namespace {

// Coefficient of the face of node i towards direction d (0..5: -z,-y,-x,+x,+y,+z),
// shared by the two nodes it joins: keyed by the lower node and the axis.
inline double face_coef(uint64_t seed, double contrast, int64_t lower, int axis) {
  return exp(contrast * (2.0 * u01(h3(seed, 40 + axis, (uint64_t)lower)) - 1.0));
}

// Row i of the weighted 7-point Laplacian on an m^3 grid with Dirichlet
// boundary faces: neighbours in ascending order, diagonal = sum of the six
// face coefficients.  put(col, value).
template <typename Put>
void laplace_row(int64_t i, int64_t m, uint64_t seed, double contrast, Put put) {
  const int64_t m2 = m * m, x = i % m, y = (i / m) % m, z = i / m2;
  // lower node and axis of each face: -z, -y, -x, +x, +y, +z
  const int64_t lo[6] = {i - m2, i - m, i - 1, i, i, i};
  const int ax[6] = {2, 1, 0, 0, 1, 2};
  const bool in[6] = {z > 0, y > 0, x > 0, x < m - 1, y < m - 1, z < m - 1};
  const int64_t nb[6] = {i - m2, i - m, i - 1, i + 1, i + m, i + m2};
  double k[6], diag = 0.0;
  for (int f = 0; f < 6; ++f) {
    // boundary faces get their own draw (lower node = -1 - i keeps the keys distinct)
    k[f] = in[f] ? face_coef(seed, contrast, lo[f], ax[f]) : face_coef(seed, contrast, -1 - i, 3 + f);
    diag += k[f];
  }
  for (int f = 0; f < 3; ++f)
    if (in[f]) put(nb[f], -k[f]);
  put(i, diag);
  for (int f = 3; f < 6; ++f)
    if (in[f]) put(nb[f], -k[f]);
}

}  // namespace

extern "C" bsp_status bsp_gen_diffusion3d(int32_t m, double contrast, uint64_t seed, int32_t *rows, int64_t *nnz,
                                          int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (m <= 0 || !rows || !nnz || !(contrast >= 0.0)) return BSP_ERR_INVALID;
  const int64_t n = (int64_t)m * m * m;
  if (n > INT32_MAX) return BSP_ERR_INVALID;
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % m, y = (i / m) % m, z = i / ((int64_t)m * m);
    cnt[i] = 1 + (x > 0) + (x < m - 1) + (y > 0) + (y < m - 1) + (z > 0) + (z < m - 1);
  }
  *rows = (int32_t)n;
  *nnz = prefix(cnt, rowPtr);
  if (!rowPtr) return BSP_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t k = rowPtr[i];
    laplace_row(i, m, seed, contrast, [&](int64_t c, double v) {
      colIdx[k] = (int32_t)c;
      values[k] = v;
      ++k;
    });
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_gen_block_laplace3d(int32_t m, int32_t dof, double cond, uint64_t seed, int32_t *rows,
                                              int64_t *nnz, int32_t *rowPtr, int32_t *colIdx, double *values) {
  if (m <= 0 || dof <= 0 || dof > 16 || !rows || !nnz || !(cond >= 1.0)) return BSP_ERR_INVALID;
  const int64_t nodes = (int64_t)m * m * m, n = nodes * dof;
  if (n > INT32_MAX) return BSP_ERR_INVALID;
  // S = Q diag(lambda) Q^T: Q from Gram-Schmidt of a seeded normal matrix,
  // lambda log-spaced in [1, cond]
  std::vector<double> Q((size_t)dof * dof), S((size_t)dof * dof, 0.0);
  for (int a = 0; a < dof * dof; ++a) Q[a] = normal(seed, 50, (uint64_t)a);
  for (int c = 0; c < dof; ++c) {
    for (int p = 0; p < c; ++p) {
      double d = 0.0;
      for (int r = 0; r < dof; ++r) d += Q[r * dof + c] * Q[r * dof + p];
      for (int r = 0; r < dof; ++r) Q[r * dof + c] -= d * Q[r * dof + p];
    }
    double nrm = 0.0;
    for (int r = 0; r < dof; ++r) nrm += Q[r * dof + c] * Q[r * dof + c];
    nrm = sqrt(nrm);
    for (int r = 0; r < dof; ++r) Q[r * dof + c] /= nrm;
  }
  for (int c = 0; c < dof; ++c) {
    const double lam = dof > 1 ? pow(cond, (double)c / (dof - 1)) : 1.0;
    for (int a = 0; a < dof; ++a)
      for (int b = 0; b < dof; ++b) S[a * dof + b] += Q[a * dof + c] * lam * Q[b * dof + c];
  }
  for (int a = 0; a < dof; ++a)  // exactly symmetric
    for (int b = 0; b < a; ++b) S[a * dof + b] = S[b * dof + a];
  std::vector<int32_t> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nodes; ++i) {
    const int64_t x = i % m, y = (i / m) % m, z = i / ((int64_t)m * m);
    const int32_t deg = 1 + (x > 0) + (x < m - 1) + (y > 0) + (y < m - 1) + (z > 0) + (z < m - 1);
    for (int a = 0; a < dof; ++a) cnt[i * dof + a] = deg * dof;
  }
  *rows = (int32_t)n;
  *nnz = prefix(cnt, rowPtr);
  if (!rowPtr) return BSP_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nodes; ++i) {
    for (int a = 0; a < dof; ++a) {
      int64_t k = rowPtr[i * dof + a];
      laplace_row(i, m, seed, 1.0, [&](int64_t c, double v) {
        for (int b = 0; b < dof; ++b) {
          colIdx[k] = (int32_t)(c * dof + b);
          values[k] = v * S[a * dof + b];
          ++k;
        }
      });
    }
  }
  return BSP_OK;
}
