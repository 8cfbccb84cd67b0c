// Batched SpMV / 8-RHS SpMM over many independent CSR matrices in one
// persistent launch.  The reference has no batched form: every operator
// wrapper handles one matrix per call (src/csrspmv.cu:104-170,
// src/spmv.cu:190-273).
//
// Plan (host, once): the row-length profile of every matrix gives
//   * its lanes per row L (the tuner: a row-statistics model, or timing of
//     the candidate L values with one launch per matrix);
//   * row items: runs of consecutive rows holding about item_nnz nonzeros,
//     processed by one warp, 32/L rows at a time; rows above 16*L nonzeros
//     inside the run are taken by the whole warp after the pass;
//   * long-row segments: rows above long_row_nnz are cut into seg_nnz pieces,
//     one warp each; a piece's partial sum goes to a slot, and the warp that
//     arrives last at the row's counter sums the slots in order and writes y
//     (the counter is reset by that warp for the next launch).
// Every output element is a fixed sum order of fixed products, whatever warp
// runs an item, so results are deterministic and identical between the
// batched launch and the per-matrix launches.
//
// Run: warps take items from a global counter; the long segments come first in
// the list so the critical path starts at time zero.  Counter reset + kernel
// are captured once in a CUDA graph.
//
// With 8 right-hand sides (x, y row-major n x 8) the lanes of a row split its
// columns into 16-byte pieces and its nonzeros as above; FP64 SELL slices
// stage their window of x rows in shared memory (see sell_item_piece).
#include <algorithm>
#include <cmath>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

struct BatchMatDev {
  const int32_t *rp;
  const int32_t *ci;
  const void *val;
  const void *x;
  void *y;
  int32_t rows, cols;
  // SELL-32 copy (null when the matrix is stored only as CSR): slice s of 32
  // rows spans entries [sell_ptr[s], sell_ptr[s + 1]); entry k of row l of
  // the slice at sell_ptr[s] + 32k + l.  Narrow form: slice rows are the
  // matrix rows in order, column = row + sell_off[entry].  Wide form: slice
  // row l of slice s is matrix row sell_perm[32s + l] (rows sorted by length
  // inside windows, rows of long segments left out), column = sell_col[entry].
  const int32_t *sell_ptr;
  const void *sell_val;
  const int16_t *sell_off;
  const int32_t *sell_perm;
  const int32_t *sell_col;
  int32_t sell_rows;
  // narrow form with several right-hand sides: per slice the lowest column
  // its entries (padding included) touch when all of them lie in a window of
  // kWinRows x rows from there, else -1; null when not built
  const int32_t *sell_lo;
};

// x rows a warp stages per SELL slice (several right-hand sides).
constexpr int kWinRows = 64;

// info == kSellItem / kSellWideItem: SELL slices [a, b) (narrow / wide form).
// info >= 0 otherwise: row item, rows [a, b), info = lanes per row.
// info < 0 : long-row segment, row a, segment b, long id = -(info + 1).
struct BatchItem {
  int32_t mat, a, b, info;
};
constexpr int32_t kSellItem = 64;
constexpr int32_t kSellWideItem = 65;

struct LongRow {
  int32_t part_base, nseg;
};

constexpr int kBatchThreads = 256;
constexpr int kMedFactor = 16;  // rows above 16*L nonzeros go to the whole warp

template <typename V, int NRHS>
struct Vec {
  V v[NRHS];
};

// x row c (NRHS consecutive values) through the read-only path.
template <typename V, int NRHS>
__device__ __forceinline__ void load_xrow(const V *__restrict__ x, int32_t c, V (&out)[NRHS]) {
  if constexpr (NRHS == 1) {
    out[0] = __ldg(x + c);
  } else if constexpr (sizeof(V) == 8) {
    const double2 *p = reinterpret_cast<const double2 *>(x + (int64_t)c * NRHS);
#pragma unroll
    for (int k = 0; k < NRHS / 2; ++k) {
      const double2 t = __ldg(p + k);
      out[2 * k] = t.x;
      out[2 * k + 1] = t.y;
    }
  } else {
    const float4 *p = reinterpret_cast<const float4 *>(x + (int64_t)c * NRHS);
#pragma unroll
    for (int k = 0; k < NRHS / 4; ++k) {
      const float4 t = __ldg(p + k);
      out[4 * k] = t.x;
      out[4 * k + 1] = t.y;
      out[4 * k + 2] = t.z;
      out[4 * k + 3] = t.w;
    }
  }
}

template <typename V, int NRHS>
__device__ __forceinline__ void fma_row(V (&acc)[NRHS], V a, const V (&xr)[NRHS]) {
#pragma unroll
  for (int k = 0; k < NRHS; ++k) acc[k] = fma(a, xr[k], acc[k]);
}

// sum over nonzeros j = s + off, s + off + stride, ... < e (4 in flight)
template <typename V, int NRHS>
__device__ __forceinline__ void strided_dot(const int32_t *__restrict__ ci, const V *__restrict__ val,
                                            const V *__restrict__ x, int32_t j, int32_t e, int32_t stride,
                                            V (&acc)[NRHS]) {
  for (; j + 3 * stride < e; j += 4 * stride) {
    int32_t c[4];
    V a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      c[u] = __ldg(ci + j + u * stride);
      a[u] = __ldg(val + j + u * stride);
    }
    V xr[4][NRHS];
#pragma unroll
    for (int u = 0; u < 4; ++u) load_xrow<V, NRHS>(x, c[u], xr[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) fma_row<V, NRHS>(acc, a[u], xr[u]);
  }
  for (; j < e; j += stride) {
    V xr[NRHS];
    load_xrow<V, NRHS>(x, __ldg(ci + j), xr);
    fma_row<V, NRHS>(acc, __ldg(val + j), xr);
  }
}

// The whole warp on one row (nonzeros [s, e)); every lane returns the sums.
template <typename V, int NRHS>
__device__ __forceinline__ void warp_row(const int32_t *ci, const V *val, const V *x, int32_t s, int32_t e,
                                         int lane, V (&acc)[NRHS]) {
#pragma unroll
  for (int k = 0; k < NRHS; ++k) acc[k] = V(0);
  strided_dot<V, NRHS>(ci, val, x, s + lane, e, 32, acc);
#pragma unroll
  for (int k = 0; k < NRHS; ++k) acc[k] = warp_sum(acc[k]);
}

template <typename V, int NRHS, int L>
__device__ __forceinline__ void rows_item(const BatchMatDev &M, int32_t r0, int32_t r1, int32_t long_thr,
                                          int lane) {
  constexpr int RPP = 32 / L;
  const int sub = lane % L, rl = lane / L;
  const V *val = static_cast<const V *>(M.val);
  const V *x = static_cast<const V *>(M.x);
  V *y = static_cast<V *>(M.y);
  // one vector: the next group's row pointers are loaded while this group's
  // entries are summed (one dependent round trip fewer per group; with 8
  // vectors the extra registers cost more than it saves)
  int32_t ns = 0, ne = 0;
  if (NRHS == 1 && r0 + rl < r1) {
    ns = __ldg(M.rp + r0 + rl);
    ne = __ldg(M.rp + r0 + rl + 1);
  }
  for (int32_t base = r0; base < r1; base += RPP) {
    const int32_t row = base + rl;
    const bool active = row < r1;
    int32_t s = 0, e = 0;
    if constexpr (NRHS == 1) {
      s = ns;
      e = ne;
      ns = ne = 0;  // a row past the item stays empty
      if (row + RPP < r1) {
        ns = __ldg(M.rp + row + RPP);
        ne = __ldg(M.rp + row + RPP + 1);
      }
    } else if (active) {
      s = __ldg(M.rp + row);
      e = __ldg(M.rp + row + 1);
    }
    const int32_t len = e - s;
    const bool mine = len <= kMedFactor * L && len <= long_thr;
    const bool medium = active && len > kMedFactor * L && len <= long_thr;
    if (!mine) e = s;  // medium rows below, long rows in their segments
    V acc[NRHS];
#pragma unroll
    for (int k = 0; k < NRHS; ++k) acc[k] = V(0);
    if constexpr (L == 1 && NRHS == 1) {
      // a lane per row: its entries in predicated groups of 4, so a short
      // row's loads go out together (same summation order)
      for (int32_t j = s; j < e; j += 4) {
        int32_t c[4];
        V a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          c[u] = j + u < e ? __ldg(M.ci + j + u) : -1;
          a[u] = j + u < e ? __ldg(val + j + u) : V(0);
        }
        V xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) xv[u] = c[u] >= 0 ? __ldg(x + c[u]) : V(0);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (c[u] >= 0) acc[0] = fma(a[u], xv[u], acc[0]);
      }
    } else {
      strided_dot<V, NRHS>(M.ci, val, x, s + sub, e, L, acc);
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1)
#pragma unroll
      for (int k = 0; k < NRHS; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (active && sub == 0 && mine) {
#pragma unroll
      for (int k = 0; k < NRHS; ++k) y[(int64_t)row * NRHS + k] = acc[k];
    }
    unsigned med = __ballot_sync(0xffffffffu, medium && sub == 0);
    while (med) {
      const int b = __ffs(med) - 1;
      med &= med - 1;
      const int32_t mrow = base + b / L;
      const int32_t ms = __ldg(M.rp + mrow), me = __ldg(M.rp + mrow + 1);
      V w[NRHS];
      warp_row<V, NRHS>(M.ci, val, x, ms, me, lane, w);
      if (lane < NRHS) {
        V o = w[0];
#pragma unroll
        for (int k = 1; k < NRHS; ++k)
          if (lane == k) o = w[k];
        y[(int64_t)mrow * NRHS + lane] = o;
      }
    }
  }
}

// SELL-32 slices [s0, s1): lane l owns slice row l and sums its entries
// in stored order, U entries' loads issued before their gathers.  Value and
// column loads of a warp are 32 consecutive entries (coalesced); for banded
// matrices (narrow form) the gathered x rows are consecutive too.
template <typename V, int NRHS, bool WIDE>
__device__ __forceinline__ void sell_item(const BatchMatDev &M, int32_t s0, int32_t s1, int lane) {
  constexpr int U = NRHS == 1 ? 4 : 2;
  const V *sv = static_cast<const V *>(M.sell_val);
  const V *x = static_cast<const V *>(M.x);
  V *y = static_cast<V *>(M.y);
  for (int32_t sl = s0; sl < s1; ++sl) {
    const int32_t pos = sl * 32 + lane;
    const bool live = pos < (WIDE ? M.sell_rows : M.rows);
    const int32_t row = WIDE ? (live ? __ldg(M.sell_perm + pos) : 0) : pos;
    const int32_t p0 = __ldg(M.sell_ptr + sl);
    const int32_t w = live ? (__ldg(M.sell_ptr + sl + 1) - p0) >> 5 : 0;
    const V *vp = sv + p0 + lane;
    const int16_t *op = M.sell_off + p0 + lane;
    const int32_t *cp = M.sell_col + p0 + lane;
    V acc[NRHS];
#pragma unroll
    for (int k = 0; k < NRHS; ++k) acc[k] = V(0);
    int32_t k = 0;
    for (; k + U <= w; k += U) {
      V a[U];
      int32_t c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        a[u] = __ldg(vp + 32 * (k + u));
        c[u] = WIDE ? __ldg(cp + 32 * (k + u)) : row + (int32_t)__ldg(op + 32 * (k + u));
      }
      V xr[U][NRHS];
#pragma unroll
      for (int u = 0; u < U; ++u) load_xrow<V, NRHS>(x, c[u], xr[u]);
#pragma unroll
      for (int u = 0; u < U; ++u) fma_row<V, NRHS>(acc, a[u], xr[u]);
    }
    for (; k < w; ++k) {
      V xr[NRHS];
      load_xrow<V, NRHS>(x, WIDE ? __ldg(cp + 32 * k) : row + (int32_t)__ldg(op + 32 * k), xr);
      fma_row<V, NRHS>(acc, __ldg(vp + 32 * k), xr);
    }
    if (live) {
#pragma unroll
      for (int j = 0; j < NRHS; ++j) y[(int64_t)row * NRHS + j] = acc[j];
    }
  }
}

// ---------------------------------------------------------------------------
// Several right-hand sides (x and y row-major, NRHS values per row): the
// CPL = NRHS * sizeof(V) / 16 lanes of a row split its columns, one 16-byte
// piece each, so a gathered x row is one contiguous access of the row's
// lanes and a lane keeps VW = 16 / sizeof(V) sums instead of NRHS (FP64, 8
// vectors: 4 lanes of 2 columns).  L lanes per row split the nonzeros as in
// the one-vector items; each column is summed in the same order as there
// (lane sub takes entries s+sub, s+sub+L, ... in order, then a fixed shuffle
// tree over the L lanes).
template <typename V> struct Piece { static constexpr int VW = 16 / (int)sizeof(V); };

template <typename V>
__device__ __forceinline__ void load_piece(const V *__restrict__ p, V (&o)[Piece<V>::VW]) {
  if constexpr (sizeof(V) == 8) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
  }
}

template <typename V>
__device__ __forceinline__ void store_piece(V *p, const V (&v)[Piece<V>::VW]) {
  if constexpr (sizeof(V) == 8)
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  else
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// acc (columns [cp*VW, cp*VW + VW)) += sum over entries j, j + stride, ... < e
// in order, in predicated groups of U: a group's entry loads go out together,
// then its U gathers together, so a short row costs one entries -> x round
// trip instead of one per entry.
template <typename V, int NRHS>
__device__ __forceinline__ void strided_piece_dot(const int32_t *__restrict__ ci, const V *__restrict__ val,
                                                  const V *__restrict__ x, int cp, int32_t j, int32_t e,
                                                  int32_t stride, V (&acc)[Piece<V>::VW]) {
  constexpr int VW = Piece<V>::VW;
  constexpr int U = 4;
  for (; j < e; j += U * stride) {
    int32_t c[U];
    V a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool ok = j + u * stride < e;
      c[u] = ok ? __ldg(ci + j + u * stride) : -1;
      a[u] = ok ? __ldg(val + j + u * stride) : V(0);
    }
    V xr[U][VW];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] >= 0) {
        load_piece<V>(x + (int64_t)c[u] * NRHS + cp * VW, xr[u]);
      } else {
#pragma unroll
        for (int k = 0; k < VW; ++k) xr[u][k] = V(0);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (c[u] >= 0) {
#pragma unroll
        for (int k = 0; k < VW; ++k) acc[k] = fma(a[u], xr[u][k], acc[k]);
      }
  }
}

// The whole warp on one row: 32 / CPL nonzero lanes; every lane returns the
// sums of its column piece.
template <typename V, int NRHS>
__device__ __forceinline__ void warp_row_piece(const int32_t *ci, const V *val, const V *x, int32_t s, int32_t e,
                                               int lane, V (&acc)[Piece<V>::VW]) {
  constexpr int VW = Piece<V>::VW;
  constexpr int CPL = NRHS / VW;
#pragma unroll
  for (int k = 0; k < VW; ++k) acc[k] = V(0);
  strided_piece_dot<V, NRHS>(ci, val, x, lane % CPL, s + lane / CPL, e, 32 / CPL, acc);
#pragma unroll
  for (int o = 16; o >= CPL; o >>= 1)
#pragma unroll
    for (int k = 0; k < VW; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
}

template <typename V, int NRHS, int L>
__device__ __forceinline__ void rows_item_piece(const BatchMatDev &M, int32_t r0, int32_t r1, int32_t long_thr,
                                                int lane) {
  constexpr int VW = Piece<V>::VW;
  constexpr int CPL = NRHS / VW;
  constexpr int LT = CPL * L;   // lanes per row
  static_assert(LT <= 32, "lanes per row");
  constexpr int RPP = 32 / LT;
  const int cp = lane % CPL, sub = (lane / CPL) % L, rl = lane / LT;
  const V *val = static_cast<const V *>(M.val);
  const V *x = static_cast<const V *>(M.x);
  V *y = static_cast<V *>(M.y);
  // the next pass's row pointers are loaded while this pass's rows are summed
  int32_t ns = 0, ne = 0;
  if (r0 + rl < r1) {
    ns = __ldg(M.rp + r0 + rl);
    ne = __ldg(M.rp + r0 + rl + 1);
  }
  for (int32_t base = r0; base < r1; base += RPP) {
    const int32_t row = base + rl;
    const bool active = row < r1;
    int32_t s = ns, e = ne;
    ns = ne = 0;
    if (row + RPP < r1) {
      ns = __ldg(M.rp + row + RPP);
      ne = __ldg(M.rp + row + RPP + 1);
    }
    const int32_t len = e - s;
    const bool mine = len <= kMedFactor * L && len <= long_thr;
    const bool medium = active && len > kMedFactor * L && len <= long_thr;
    if (!mine) e = s;
    V acc[VW];
#pragma unroll
    for (int k = 0; k < VW; ++k) acc[k] = V(0);
    strided_piece_dot<V, NRHS>(M.ci, val, x, cp, s + sub, e, L, acc);
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1)
#pragma unroll
      for (int k = 0; k < VW; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o * CPL);
    if (active && sub == 0 && mine) store_piece<V>(y + (int64_t)row * NRHS + cp * VW, acc);
    unsigned med = __ballot_sync(0xffffffffu, medium && sub == 0 && cp == 0);
    while (med) {
      const int b = __ffs(med) - 1;
      med &= med - 1;
      const int32_t mrow = base + b / LT;
      const int32_t ms = __ldg(M.rp + mrow), me = __ldg(M.rp + mrow + 1);
      V w[VW];
      warp_row_piece<V, NRHS>(M.ci, val, x, ms, me, lane, w);
      if (lane < CPL) store_piece<V>(y + (int64_t)mrow * NRHS + lane * VW, w);
    }
  }
}

// SELL-32 slices with several right-hand sides: a pass takes 32 / CPL of the
// slice's rows, CPL lanes each; every row's entries in stored order.
//
// A narrow-form slice whose entries all lie in kWinRows x rows from
// sell_lo[slice] (banded matrices) first copies that window of x into the
// warp's shared-memory buffer `xw` (kWinRows * NRHS values, coalesced
// 16-byte loads) and gathers from there: the 32 rows' overlapping x rows are
// read once per slice instead of once per entry, and each entry's gather no
// longer waits on L1/L2.  The arithmetic and its order are unchanged.
template <typename V, int NRHS>
__device__ __forceinline__ void fetch_piece(const V *__restrict__ x, const V *xw, int32_t lo, int32_t c, int cp,
                                            V (&o)[Piece<V>::VW]) {
  constexpr int VW = Piece<V>::VW;
  if (lo >= 0) {
    const V *p = xw + (c - lo) * NRHS + cp * VW;
    if constexpr (VW == 2) {
      const double2 t = *reinterpret_cast<const double2 *>(p);
      o[0] = t.x;
      o[1] = t.y;
    } else {
      const float4 t = *reinterpret_cast<const float4 *>(p);
      o[0] = t.x;
      o[1] = t.y;
      o[2] = t.z;
      o[3] = t.w;
    }
  } else {
    load_piece<V>(x + (int64_t)c * NRHS + cp * VW, o);
  }
}

template <typename V, int NRHS, bool WIDE>
__device__ __forceinline__ void sell_item_piece(const BatchMatDev &M, int32_t s0, int32_t s1, int lane, V *xw) {
  constexpr int VW = Piece<V>::VW;
  constexpr int CPL = NRHS / VW;
  constexpr int RPP = 32 / CPL;
  constexpr int U = 4;
  const int cp = lane % CPL;
  const V *sv = static_cast<const V *>(M.sell_val);
  const V *x = static_cast<const V *>(M.x);
  V *y = static_cast<V *>(M.y);
  for (int32_t sl = s0; sl < s1; ++sl) {
    const int32_t p0 = __ldg(M.sell_ptr + sl);
    const int32_t w = (__ldg(M.sell_ptr + sl + 1) - p0) >> 5;
    const int32_t lo = (!WIDE && M.sell_lo) ? __ldg(M.sell_lo + sl) : -1;   // warp-uniform
    if (lo >= 0) {
      __syncwarp();   // the previous slice's reads of xw are done
      for (int t = lane; t < kWinRows * CPL; t += 32) {
        const int32_t r = lo + t / CPL;
        if (r < M.cols) {
          V v[VW];
          load_piece<V>(x + (int64_t)r * NRHS + (t % CPL) * VW, v);
          store_piece<V>(xw + t * VW, v);
        }
      }
      __syncwarp();
    }
    for (int q = 0; q < CPL; ++q) {
      const int l = q * RPP + lane / CPL;   // slice row
      const int32_t pos = sl * 32 + l;
      const bool live = pos < (WIDE ? M.sell_rows : M.rows);
      const int32_t row = WIDE ? (live ? __ldg(M.sell_perm + pos) : 0) : pos;
      const int32_t wl = live ? w : 0;
      const V *vp = sv + p0 + l;
      const int16_t *op = M.sell_off + p0 + l;
      const int32_t *cpp = M.sell_col + p0 + l;
      V acc[VW];
#pragma unroll
      for (int k = 0; k < VW; ++k) acc[k] = V(0);
      for (int32_t k = 0; k < wl; k += U) {   // predicated groups of U, entries in stored order
        V a[U];
        int32_t c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool ok = k + u < wl;
          a[u] = ok ? __ldg(vp + 32 * (k + u)) : V(0);
          c[u] = !ok ? -1 : WIDE ? __ldg(cpp + 32 * (k + u)) : row + (int32_t)__ldg(op + 32 * (k + u));
        }
        V xr[U][VW];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (c[u] >= 0) {
            fetch_piece<V, NRHS>(x, xw, lo, c[u], cp, xr[u]);
          } else {
#pragma unroll
            for (int t = 0; t < VW; ++t) xr[u][t] = V(0);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (c[u] >= 0) {
#pragma unroll
            for (int t = 0; t < VW; ++t) acc[t] = fma(a[u], xr[u][t], acc[t]);
          }
      }
      if (live) store_piece<V>(y + (int64_t)row * NRHS + cp * VW, acc);
    }
  }
}

// Fills the SELL-32 copy of one matrix: thread per row; padding entries get
// value 0 and the column min(row, cols - 1).  *bad is set when a column
// lies 32768 or more from its row.
template <typename V>
__global__ void batch_sell_fill_kernel(int32_t rows, int32_t cols, const int32_t *__restrict__ rp,
                                       const int32_t *__restrict__ ci, const V *__restrict__ val,
                                       const int32_t *__restrict__ sptr, V *__restrict__ sval,
                                       int16_t *__restrict__ soff, int32_t *__restrict__ bad) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sl = (int32_t)(r >> 5), l = (int32_t)(r & 31);
    const int32_t p0 = sptr[sl], w = (sptr[sl + 1] - p0) >> 5;
    const int32_t s = rp[r], len = rp[r + 1] - s;
    const int32_t pc = (int32_t)(r < (int64_t)cols - 1 ? r : (int64_t)cols - 1);
    for (int32_t k = 0; k < w; ++k) {
      const bool real = k < len;
      const int64_t d = (int64_t)(real ? ci[s + k] : pc) - r;
      if (d < -32768 || d > 32767) atomicExch(bad, 1);
      sval[p0 + 32 * k + l] = real ? val[s + k] : V(0);
      soff[p0 + 32 * k + l] = (int16_t)(d < -32768 || d > 32767 ? 0 : d);
    }
  }
}

// Fills the wide SELL-32 copy: thread per slice row; slice row p is matrix
// row perm[p]; padding entries get value 0 and column 0.
template <typename V>
__global__ void batch_sell_fill_wide_kernel(int32_t nrows, const int32_t *__restrict__ perm,
                                            const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                            const V *__restrict__ val, const int32_t *__restrict__ sptr,
                                            V *__restrict__ sval, int32_t *__restrict__ scol) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nrows; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sl = (int32_t)(p >> 5), l = (int32_t)(p & 31);
    const int32_t p0 = sptr[sl], w = (sptr[sl + 1] - p0) >> 5;
    const int32_t r = perm[p];
    const int32_t s = rp[r], len = rp[r + 1] - s;
    for (int32_t k = 0; k < w; ++k) {
      const bool real = k < len;
      sval[p0 + 32 * k + l] = real ? val[s + k] : V(0);
      scol[p0 + 32 * k + l] = real ? ci[s + k] : 0;
    }
  }
}

// Per narrow SELL slice: the lowest column its 32 rows' stored entries read
// (a padding entry of row r reads column min(r, cols - 1)), or -1 when they
// span kWinRows or more columns.  Thread per row, a warp per slice (the loop
// bound is rounded up to whole warps so every lane reaches the reductions).
__global__ void batch_sell_window_kernel(int32_t rows, int32_t cols, const int32_t *__restrict__ rp,
                                         const int32_t *__restrict__ ci, int32_t *__restrict__ lo_out) {
  const int64_t n = ((int64_t)rows + 31) / 32 * 32;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    int32_t mn = INT32_MAX, mx = INT32_MIN;
    if (r < rows) {
      mn = mx = (int32_t)(r < (int64_t)cols - 1 ? r : (int64_t)cols - 1);
      for (int32_t j = rp[r]; j < rp[r + 1]; ++j) {
        const int32_t c = ci[j];
        mn = min(mn, c);
        mx = max(mx, c);
      }
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((r & 31) == 0) lo_out[r >> 5] = (int64_t)mx - mn < kWinRows ? mn : -1;
  }
}

template <typename V, int NRHS>
__device__ __forceinline__ void segment_item(const BatchMatDev &M, int32_t row, int32_t seg, int32_t lid,
                                             int32_t seg_nnz, const LongRow *__restrict__ longs,
                                             V *__restrict__ part, int32_t *__restrict__ arrive, int lane) {
  const V *val = static_cast<const V *>(M.val);
  const V *x = static_cast<const V *>(M.x);
  const LongRow lr = longs[lid];
  const int32_t s0 = __ldg(M.rp + row), e0 = __ldg(M.rp + row + 1);
  const int32_t s = s0 + seg * seg_nnz;
  const int32_t e = min(s + seg_nnz, e0);
  if constexpr (NRHS > 1) {
    constexpr int VW = Piece<V>::VW;
    V w[VW];
    warp_row_piece<V, NRHS>(M.ci, val, x, s, e, lane, w);
    if (lane < NRHS / VW) {
      store_piece<V>(part + (int64_t)(lr.part_base + seg) * NRHS + lane * VW, w);
      __threadfence();
    }
  } else {
    V w[1];
    warp_row<V, 1>(M.ci, val, x, s, e, lane, w);
    if (lane == 0) {
      part[lr.part_base + seg] = w[0];
      __threadfence();
    }
  }
  __syncwarp();
  int last = 0;
  if (lane == 0) last = atomicAdd(arrive + lid, 1) == lr.nseg - 1;
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();
  if (lane < NRHS) {
    V acc = V(0);
    for (int32_t t = 0; t < lr.nseg; ++t) acc += __ldcg(part + (int64_t)(lr.part_base + t) * NRHS + lane);
    static_cast<V *>(M.y)[(int64_t)row * NRHS + lane] = acc;
  }
  if (lane == 0) atomicExch(arrive + lid, 0);  // ready for the next launch
}

// One FP32 vector: capped at 40 registers (6 resident CTAs per SM).  At 32
// registers (8 CTAs) it was faster before the SELL items joined the kernel
// (222.5 -> 204.5 us) but now spills there, and 6 CTAs measured faster
// (512-matrix batch, tuned: 190.7 -> 174.1 us).  FP64 and the 8-vector forms
// keep the compiler's choice.
template <typename V, int NRHS>
__global__ void __launch_bounds__(kBatchThreads, (NRHS == 1 && sizeof(V) == 4) ? 6 : 0) batch_kernel(const BatchMatDev *__restrict__ mats,
                                                              const BatchItem *__restrict__ items, int32_t nitems,
                                                              int32_t *__restrict__ next,
                                                              const LongRow *__restrict__ longs,
                                                              V *__restrict__ part, int32_t *__restrict__ arrive,
                                                              int32_t seg_nnz, int32_t long_thr) {
  const int lane = threadIdx.x & 31;
  constexpr bool kWin = NRHS > 1 && sizeof(V) == 8;
  __shared__ __align__(16) V xwin[kWin ? (kBatchThreads / 32) * kWinRows * NRHS : 1];
  V *xw = xwin + (kWin ? (threadIdx.x >> 5) * kWinRows * NRHS : 0);
  for (;;) {
    int32_t it = 0;
    if (lane == 0) it = atomicAdd(next, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= nitems) return;
    const BatchItem I = items[it];
    const BatchMatDev M = mats[I.mat];
    // SELL slices with several FP64 right-hand sides: column pieces and the
    // shared-memory x window (512-matrix batch, banded half, 8 vectors: 517 ->
    // 371 us); FP32 keeps a lane per row over all columns there (197 us
    // against 224 us in pieces)
    if (I.info == kSellItem) {
      if constexpr (NRHS > 1 && sizeof(V) == 8)
        sell_item_piece<V, NRHS, false>(M, I.a, I.b, lane, xw);
      else
        sell_item<V, NRHS, false>(M, I.a, I.b, lane);
      continue;
    }
    if (I.info == kSellWideItem) {
      if constexpr (NRHS > 1 && sizeof(V) == 8)
        sell_item_piece<V, NRHS, true>(M, I.a, I.b, lane, xw);
      else
        sell_item<V, NRHS, true>(M, I.a, I.b, lane);
      continue;
    }
    if (I.info < 0) {
      segment_item<V, NRHS>(M, I.a, I.b, -(I.info + 1), seg_nnz, longs, part, arrive, lane);
      continue;
    }
    if constexpr (NRHS > 1) {
      // lanes per row split the nonzeros; at most 32 / CPL of them
      constexpr int LMAX = 32 / (NRHS / Piece<V>::VW);
      const int32_t L = I.info < LMAX ? I.info : LMAX;
      switch (L) {
        case 1: rows_item_piece<V, NRHS, 1>(M, I.a, I.b, long_thr, lane); break;
        case 2: rows_item_piece<V, NRHS, 2>(M, I.a, I.b, long_thr, lane); break;
        case 4: rows_item_piece<V, NRHS, 4>(M, I.a, I.b, long_thr, lane); break;
        case 8: rows_item_piece<V, NRHS, (LMAX >= 8 ? 8 : LMAX)>(M, I.a, I.b, long_thr, lane); break;
        default: rows_item_piece<V, NRHS, LMAX>(M, I.a, I.b, long_thr, lane); break;
      }
    } else {
      switch (I.info) {
        case 1: rows_item<V, NRHS, 1>(M, I.a, I.b, long_thr, lane); break;
        case 2: rows_item<V, NRHS, 2>(M, I.a, I.b, long_thr, lane); break;
        case 4: rows_item<V, NRHS, 4>(M, I.a, I.b, long_thr, lane); break;
        case 8: rows_item<V, NRHS, 8>(M, I.a, I.b, long_thr, lane); break;
        case 16: rows_item<V, NRHS, 16>(M, I.a, I.b, long_thr, lane); break;
        default: rows_item<V, NRHS, 32>(M, I.a, I.b, long_thr, lane); break;
      }
    }
  }
}

}  // namespace bsp

using namespace bsp;

struct bsp_batch_plan_s {
  int32_t count = 0, nrhs = 1;
  bsp_dtype dtype = BSP_F64;
  bsp_batch_options opt{};
  std::vector<bsp_batch_mat> host_mats;
  std::vector<std::vector<int32_t>> lens;  // row lengths per matrix
  std::vector<int32_t> lanes;
  std::vector<int32_t> fmt;                 // 0 CSR, 1 SELL-32 narrow, 2 SELL-32 wide
  std::vector<uint8_t> sell_ok;             // 0 none, 1 narrow, 2 wide copy built
  std::vector<std::vector<int32_t>> sell_slices;  // slice pointers (host copy)
  std::vector<int32_t> sell_T;              // wide form: rows above this go to segments
  std::vector<BatchMatDev> dm;              // host copy of the descriptors
  void *d_sell_val = nullptr;
  int16_t *d_sell_off = nullptr;
  int32_t *d_sell_ptr = nullptr;
  int32_t *d_sell_col = nullptr;
  int32_t *d_sell_perm = nullptr;
  int32_t *d_sell_lo = nullptr;
  BatchMatDev *d_mats = nullptr;
  // batched list (long segments first) and per-matrix lists
  BatchItem *d_items = nullptr, *d_items_sep = nullptr;
  int64_t nitems = 0;
  std::vector<int64_t> sep_off;  // [count+1] offsets into d_items_sep
  LongRow *d_longs = nullptr;
  int64_t nlong = 0, nseg = 0, total_nnz = 0;
  void *d_part = nullptr;
  int32_t *d_arrive = nullptr;
  int32_t *d_next = nullptr;  // [count + 1]: batched counter, then one per matrix
  int grid = 0;
  cudaStream_t graph_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
};

namespace {

int model_lanes(const std::vector<int32_t> &len, int32_t long_thr, int nrhs) {
  double s = 0;
  int64_t n = 0;
  for (int32_t l : len)
    if (l <= long_thr) {
      s += l;
      ++n;
    }
  const double mean = n ? s / (double)n : 0.0;
  const double per_lane = nrhs > 1 ? 2.0 : 4.0;  // nonzeros a lane should own
  int L = 1;
  while (L < 32 && (double)L * per_lane < mean) L <<= 1;
  return mean <= 2.0 * per_lane ? 1 : L;
}

// SELL-32 slice pointers of a matrix from its row lengths; empty when the
// padding would add more than 1/8 to the entries, a row is longer than
// long_thr, or the padded size passes 2^31.
std::vector<int32_t> sell_slices(const std::vector<int32_t> &len, int32_t long_thr) {
  const int64_t n = (int64_t)len.size();
  const int64_t ns = (n + 31) / 32;
  std::vector<int32_t> ptr((size_t)ns + 1, 0);
  int64_t nnz = 0, acc = 0;
  for (int64_t sl = 0; sl < ns; ++sl) {
    int32_t w = 0;
    for (int64_t r = sl * 32; r < std::min(n, sl * 32 + 32); ++r) {
      if (len[r] > long_thr) return {};
      w = std::max(w, len[r]);
      nnz += len[r];
    }
    acc += 32 * (int64_t)w;
    if (acc >= INT32_MAX) return {};
    ptr[sl + 1] = (int32_t)acc;
  }
  if (n == 0 || 8 * acc > 9 * nnz) return {};
  return ptr;
}

// Wide SELL-32 layout: the rows of at most T entries sorted by length
// (longest first, stable) and cut into slices of 32; `perm` gets the slice
// rows' matrix rows, *T_out the cut.  T is the largest power of two <=
// long_thr (down to 8) whose padding adds at most 1/8 to those rows'
// entries; the rows above T are taken by whole warps as segments.  On the
// batch's Zipf(2.2) matrices a full sort pads by a median 3% at T = 32,
// where sorting inside windows of 1024 rows padded by 29%.  Empty when no T
// qualifies or the padded size passes 2^31.
std::vector<int32_t> sell_slices_wide(const std::vector<int32_t> &len, int32_t long_thr, std::vector<int32_t> &perm,
                                      int32_t *T_out) {
  std::vector<int32_t> order(len.size());
  for (size_t r = 0; r < len.size(); ++r) order[r] = (int32_t)r;
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return len[a] > len[b]; });
  int32_t T = 8;
  while (T * 2 <= long_thr) T *= 2;
  for (; T >= 8; T /= 2) {
    // rows of at most T entries: a suffix of the sorted order
    size_t first = 0;
    while (first < order.size() && len[order[first]] > T) ++first;
    const int64_t n = (int64_t)(order.size() - first);
    if (n == 0) continue;
    const int64_t ns = (n + 31) / 32;
    std::vector<int32_t> ptr((size_t)ns + 1, 0);
    int64_t nnz = 0, acc = 0;
    bool fits = true;
    for (int64_t sl = 0; sl < ns && fits; ++sl) {
      const int32_t w = len[order[first + sl * 32]];   // longest of the slice
      for (int64_t p = sl * 32; p < std::min(n, sl * 32 + 32); ++p) nnz += len[order[first + p]];
      acc += 32 * (int64_t)w;
      if (acc >= INT32_MAX) fits = false;
      else ptr[sl + 1] = (int32_t)acc;
    }
    if (!fits || 8 * acc > 9 * nnz) continue;
    perm.assign(order.begin() + first, order.end());
    *T_out = T;
    return ptr;
  }
  perm.clear();
  return {};
}

// Items of a SELL-32 matrix: runs of slices costing about item_nnz, a
// slice costing its entries plus 64 (its rows' overhead, as the CSR row
// items count 2 per row): slices of one-entry rows would otherwise pile
// dozens of dependent slice walks on one warp.
void build_sell_items(int32_t m, const std::vector<int32_t> &sptr, int64_t item_nnz, int32_t info,
                      std::vector<BatchItem> &out) {
  const int32_t ns = (int32_t)sptr.size() - 1;
  int32_t s0 = 0;
  int64_t acc = 0;
  for (int32_t sl = 0; sl < ns; ++sl) {
    acc += (int64_t)sptr[sl + 1] - sptr[sl] + 64;
    if (acc >= item_nnz || sl + 1 == ns) {
      out.push_back({m, s0, sl + 1, info});
      s0 = sl + 1;
      acc = 0;
    }
  }
}

// Items of matrix m for lanes L: long segments (appended to `lng`, with
// their long-row entries), then row items (to `rows`).
void build_items(int32_t m, const std::vector<int32_t> &len, int L, const bsp_batch_options &o,
                 std::vector<BatchItem> &lng, std::vector<BatchItem> &rows, std::vector<LongRow> &longs,
                 int64_t &parts, int64_t item_nnz, int32_t long_only_thr = -1) {
  const int32_t n = (int32_t)len.size();
  const int32_t thr = long_only_thr >= 0 ? long_only_thr : o.long_row_nnz;
  for (int32_t r = 0; r < n; ++r)
    if (len[r] > thr) {
      const int32_t ns = (len[r] + o.seg_nnz - 1) / o.seg_nnz;
      const int32_t lid = (int32_t)longs.size();
      longs.push_back({(int32_t)parts, ns});
      parts += ns;
      for (int32_t s = 0; s < ns; ++s) lng.push_back({m, r, s, -(lid + 1)});
    }
  if (long_only_thr >= 0) return;
  const int64_t max_rows = (int64_t)(32 / L) * 256;
  int32_t r0 = 0;
  int64_t acc = 0;
  for (int32_t r = 0; r < n; ++r) {
    acc += (len[r] <= o.long_row_nnz ? len[r] : 0) + 2;  // a row costs ~2 nonzeros of overhead
    if (acc >= item_nnz || r + 1 - r0 >= max_rows) {
      rows.push_back({m, r0, r + 1, L});
      r0 = r + 1;
      acc = 0;
    }
  }
  if (r0 < n) rows.push_back({m, r0, n, L});
}

}  // namespace

static bsp_status batch_build(bsp_batch_plan P, cudaStream_t s);
static bsp_status batch_launch_one(bsp_batch_plan P, int32_t m, cudaStream_t s);

extern "C" bsp_status bsp_batch_default_options(bsp_batch_options *o) {
  clear_error();
  BSP_CHECK_ARG(o, "null pointer");
  o->tune = 0;
  // 512-matrix batch (tuned): 1024 / 512 against 2048 / 1024 measured FP64
  // 8 vectors 652.1 -> 635.7 us, FP32 8 vectors 351.6 -> 349.5 us, one vector
  // 200.8 -> 199.7 / 160.6 -> 159.2 us; 512 / 256 and below no better
  o->seg_nnz = 512;
  o->long_row_nnz = 1024;
  o->item_nnz = 0;
  o->use_graph = 1;
  o->sell = 1;
  o->sell_wide = 0;
  return BSP_OK;
}

template <typename V, int NRHS>
static bsp_status launch_batch(bsp_batch_plan P, const BatchItem *items, int64_t nitems, int32_t *next,
                               int grid, cudaStream_t s) {
  batch_kernel<V, NRHS><<<grid, kBatchThreads, 0, s>>>(P->d_mats, items, (int32_t)nitems, next, P->d_longs,
                                                       static_cast<V *>(P->d_part), P->d_arrive, P->opt.seg_nnz,
                                                       P->opt.long_row_nnz);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

static bsp_status dispatch(bsp_batch_plan P, const BatchItem *items, int64_t nitems, int32_t *next, int grid,
                           cudaStream_t s) {
  if (nitems == 0) return BSP_OK;
  if (P->dtype == BSP_F64)
    return P->nrhs == 8 ? launch_batch<double, 8>(P, items, nitems, next, grid, s)
                        : launch_batch<double, 1>(P, items, nitems, next, grid, s);
  return P->nrhs == 8 ? launch_batch<float, 8>(P, items, nitems, next, grid, s)
                      : launch_batch<float, 1>(P, items, nitems, next, grid, s);
}

template <typename V, int NRHS>
static int occupancy() {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel<V, NRHS>, kBatchThreads, 0) != cudaSuccess ||
      b < 1)
    b = 1;
  return b;
}

static bsp_status batch_build(bsp_batch_plan P, cudaStream_t s) {
  const bsp_batch_options &o = P->opt;
  std::vector<BatchItem> lng, rows, sep;
  std::vector<LongRow> longs;
  int64_t parts = 0;
  int64_t item_nnz = o.item_nnz;
  const int warps_per_cta = kBatchThreads / 32;
  int occ = 1;
  if (P->dtype == BSP_F64)
    occ = P->nrhs == 8 ? occupancy<double, 8>() : occupancy<double, 1>();
  else
    occ = P->nrhs == 8 ? occupancy<float, 8>() : occupancy<float, 1>();
  P->grid = sm_count() * occ;
  if (item_nnz <= 0) {
    const int64_t warps = (int64_t)P->grid * warps_per_cta;
    item_nnz = P->total_nnz / (warps * 6);
    item_nnz = std::max<int64_t>(256, std::min<int64_t>(item_nnz, 8192));
    if (P->nrhs == 8) item_nnz = std::max<int64_t>(128, item_nnz / 4);
  }
  P->sep_off.assign(P->count + 1, 0);
  for (int32_t m = 0; m < P->count; ++m) {
    std::vector<BatchItem> l1, r1;
    if (P->fmt[m] == 1) {
      build_sell_items(m, P->sell_slices[m], item_nnz, kSellItem, r1);
    } else if (P->fmt[m] == 2) {   // long rows as segments, the rest from the wide copy
      build_items(m, P->lens[m], P->lanes[m], o, l1, r1, longs, parts, item_nnz, P->sell_T[m]);
      build_sell_items(m, P->sell_slices[m], item_nnz, kSellWideItem, r1);
    } else {
      build_items(m, P->lens[m], P->lanes[m], o, l1, r1, longs, parts, item_nnz);
    }
    lng.insert(lng.end(), l1.begin(), l1.end());
    rows.insert(rows.end(), r1.begin(), r1.end());
    sep.insert(sep.end(), l1.begin(), l1.end());
    sep.insert(sep.end(), r1.begin(), r1.end());
    P->sep_off[m + 1] = (int64_t)sep.size();
  }
  std::vector<BatchItem> all(lng);
  all.insert(all.end(), rows.begin(), rows.end());
  BSP_CHECK_ARG(all.size() < (size_t)INT32_MAX, "too many work items");
  P->nitems = (int64_t)all.size();
  P->nlong = (int64_t)longs.size();
  P->nseg = (int64_t)lng.size();
  dfree(P->d_items, s);
  dfree(P->d_items_sep, s);
  dfree(P->d_longs, s);
  dfree(P->d_arrive, s);
  if (P->d_part) cudaFreeAsync(P->d_part, s);
  P->d_part = nullptr;
  BSP_TRY(dalloc(&P->d_items, all.size(), s));
  BSP_TRY(dalloc(&P->d_items_sep, sep.size(), s));
  BSP_TRY(dalloc(&P->d_longs, longs.size(), s));
  BSP_TRY(dalloc(&P->d_arrive, longs.size(), s));
  const size_t es = P->dtype == BSP_F64 ? 8 : 4;
  BSP_CUDA(cudaMallocAsync(&P->d_part, (size_t)std::max<int64_t>(1, parts) * P->nrhs * es, s));
  if (!all.empty())
    BSP_CUDA(cudaMemcpyAsync(P->d_items, all.data(), all.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
  if (!sep.empty())
    BSP_CUDA(
        cudaMemcpyAsync(P->d_items_sep, sep.data(), sep.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, s));
  if (!longs.empty()) {
    BSP_CUDA(cudaMemcpyAsync(P->d_longs, longs.data(), longs.size() * sizeof(LongRow), cudaMemcpyHostToDevice, s));
    BSP_CUDA(cudaMemsetAsync(P->d_arrive, 0, longs.size() * sizeof(int32_t), s));
  }
  BSP_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
  return BSP_OK;
}

static bsp_status batch_launch_one(bsp_batch_plan P, int32_t m, cudaStream_t s) {
  const int64_t a = P->sep_off[m], b = P->sep_off[m + 1];
  if (b == a) return BSP_OK;
  const int warps_per_cta = kBatchThreads / 32;
  int grid = (int)std::min<int64_t>(ceil_div(b - a, warps_per_cta), (int64_t)P->grid);
  BSP_CUDA(cudaMemsetAsync(P->d_next + 1 + m, 0, sizeof(int32_t), s));
  return dispatch(P, P->d_items_sep + a, b - a, P->d_next + 1 + m, grid, s);
}

static bsp_status capture(bsp_batch_plan P) {
  if (P->graph) {
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  if (!P->opt.use_graph) return BSP_OK;
  if (!P->graph_stream) BSP_CUDA(cudaStreamCreateWithFlags(&P->graph_stream, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  BSP_CUDA(cudaStreamBeginCapture(P->graph_stream, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(P->d_next, 0, sizeof(int32_t), P->graph_stream);
  const bsp_status st = dispatch(P, P->d_items, P->nitems, P->d_next, P->grid, P->graph_stream);
  cudaError_t e = cudaStreamEndCapture(P->graph_stream, &g);
  if (st != BSP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  BSP_CUDA(e);
  e = cudaGraphInstantiate(&P->graph, g, 0);
  cudaGraphDestroy(g);
  BSP_CUDA(e);
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_destroy(bsp_batch_plan P) {
  clear_error();
  if (!P) return BSP_OK;
  cudaStream_t s = 0;
  if (P->graph) cudaGraphExecDestroy(P->graph);
  if (P->graph_stream) cudaStreamDestroy(P->graph_stream);
  dfree(P->d_mats, s);
  dfree(P->d_items, s);
  dfree(P->d_items_sep, s);
  dfree(P->d_longs, s);
  dfree(P->d_arrive, s);
  dfree(P->d_next, s);
  if (P->d_part) cudaFreeAsync(P->d_part, s);
  if (P->d_sell_val) cudaFreeAsync(P->d_sell_val, s);
  dfree(P->d_sell_off, s);
  dfree(P->d_sell_ptr, s);
  dfree(P->d_sell_lo, s);
  dfree(P->d_sell_col, s);
  dfree(P->d_sell_perm, s);
  cudaStreamSynchronize(s);
  delete P;
  return BSP_OK;
}

namespace {
// Builds the SELL-32 copies (one allocation per array kind for all
// matrices) and fills P->sell_ok: the narrow form (rows in order, 16-bit
// offsets) where it qualifies, else the wide form (rows sorted by length in
// windows, 32-bit columns, long rows left to segments) where its padding
// qualifies.  A narrow copy whose offsets turn out not to fit int16 is
// dropped and the matrix stays CSR.
bsp_status build_sell(bsp_batch_plan P, cudaStream_t s) {
  const int32_t count = P->count;
  P->sell_ok.assign(count, 0);
  P->sell_slices.assign(count, {});
  P->sell_T.assign(count, 0);
  if (!P->opt.sell) return BSP_OK;
  std::vector<std::vector<int32_t>> perms(count);
  int64_t tot_val = 0, tot_narrow = 0, tot_wide = 0, tot_ptr = 0, tot_perm = 0;
  std::vector<int64_t> val_off(count, 0), off_off(count, 0), col_off(count, 0), ptr_off(count, 0), perm_off(count, 0);
  for (int32_t m = 0; m < count; ++m) {
    if (P->host_mats[m].cols <= 0) continue;
    std::vector<int32_t> sp = sell_slices(P->lens[m], P->opt.long_row_nnz);
    uint8_t kind = 1;
    if (sp.empty() && P->opt.sell_wide) {
      sp = sell_slices_wide(P->lens[m], P->opt.long_row_nnz, perms[m], &P->sell_T[m]);
      kind = 2;
    }
    if (sp.empty()) continue;
    const int64_t ent = sp.back();
    val_off[m] = tot_val;
    tot_val += ent;
    if (kind == 1) {
      off_off[m] = tot_narrow;
      tot_narrow += ent;
    } else {
      col_off[m] = tot_wide;
      tot_wide += ent;
      perm_off[m] = tot_perm;
      tot_perm += (int64_t)perms[m].size();
    }
    ptr_off[m] = tot_ptr;
    tot_ptr += (int64_t)sp.size();
    P->sell_slices[m] = std::move(sp);
    P->sell_ok[m] = kind;
  }
  if (tot_ptr == 0) return BSP_OK;
  const size_t es = P->dtype == BSP_F64 ? 8 : 4;
  BSP_CUDA(cudaMallocAsync(&P->d_sell_val, (size_t)std::max<int64_t>(tot_val, 1) * es, s));
  BSP_TRY(dalloc(&P->d_sell_off, (size_t)std::max<int64_t>(tot_narrow, 1), s));
  BSP_TRY(dalloc(&P->d_sell_col, (size_t)std::max<int64_t>(tot_wide, 1), s));
  BSP_TRY(dalloc(&P->d_sell_perm, (size_t)std::max<int64_t>(tot_perm, 1), s));
  BSP_TRY(dalloc(&P->d_sell_ptr, (size_t)tot_ptr, s));
  if (P->nrhs > 1 && P->dtype == BSP_F64) BSP_TRY(dalloc(&P->d_sell_lo, (size_t)tot_ptr, s));
  int32_t *bad = nullptr;
  BSP_TRY(dalloc(&bad, (size_t)count, s));
  BSP_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t) * count, s));
  BSP_CUDA(cudaMemsetAsync(P->d_sell_val, 0, (size_t)std::max<int64_t>(tot_val, 1) * es, s));
  BSP_CUDA(cudaMemsetAsync(P->d_sell_off, 0, sizeof(int16_t) * (size_t)std::max<int64_t>(tot_narrow, 1), s));
  BSP_CUDA(cudaMemsetAsync(P->d_sell_col, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(tot_wide, 1), s));
  for (int32_t m = 0; m < count; ++m) {
    if (!P->sell_ok[m]) continue;
    const std::vector<int32_t> &sp = P->sell_slices[m];
    int32_t *dptr = P->d_sell_ptr + ptr_off[m];
    BSP_CUDA(cudaMemcpyAsync(dptr, sp.data(), sp.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const bsp_batch_mat &A = P->host_mats[m];
    void *v = static_cast<char *>(P->d_sell_val) + val_off[m] * (int64_t)es;
    if (P->sell_ok[m] == 1) {
      const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(A.rows, 256), 4096));
      int16_t *off = P->d_sell_off + off_off[m];
      if (P->dtype == BSP_F64)
        batch_sell_fill_kernel<double><<<grid, 256, 0, s>>>(A.rows, A.cols, A.rowPtr, A.colIdx,
                                                            static_cast<const double *>(A.values), dptr,
                                                            static_cast<double *>(v), off, bad + m);
      else
        batch_sell_fill_kernel<float><<<grid, 256, 0, s>>>(A.rows, A.cols, A.rowPtr, A.colIdx,
                                                           static_cast<const float *>(A.values), dptr,
                                                           static_cast<float *>(v), off, bad + m);
      P->dm[m].sell_off = off;
      P->dm[m].sell_rows = A.rows;
      if (P->d_sell_lo) {
        int32_t *lo = P->d_sell_lo + ptr_off[m];
        batch_sell_window_kernel<<<grid, 256, 0, s>>>(A.rows, A.cols, A.rowPtr, A.colIdx, lo);
        BSP_LAUNCH_CHECK();
        P->dm[m].sell_lo = lo;
      }
    } else {
      const int32_t nr = (int32_t)perms[m].size();
      int32_t *perm = P->d_sell_perm + perm_off[m];
      int32_t *col = P->d_sell_col + col_off[m];
      BSP_CUDA(cudaMemcpyAsync(perm, perms[m].data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice, s));
      const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(nr, 256), 4096));
      if (P->dtype == BSP_F64)
        batch_sell_fill_wide_kernel<double><<<grid, 256, 0, s>>>(nr, perm, A.rowPtr, A.colIdx,
                                                                 static_cast<const double *>(A.values), dptr,
                                                                 static_cast<double *>(v), col);
      else
        batch_sell_fill_wide_kernel<float><<<grid, 256, 0, s>>>(nr, perm, A.rowPtr, A.colIdx,
                                                                static_cast<const float *>(A.values), dptr,
                                                                static_cast<float *>(v), col);
      P->dm[m].sell_perm = perm;
      P->dm[m].sell_col = col;
      P->dm[m].sell_rows = nr;
    }
    BSP_LAUNCH_CHECK();
    P->dm[m].sell_ptr = dptr;
    P->dm[m].sell_val = v;
  }
  // host vectors (slice pointers, permutations) stay alive until this sync
  std::vector<int32_t> hbad(count, 0);
  BSP_CUDA(cudaMemcpyAsync(hbad.data(), bad, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  dfree(bad, s);
  for (int32_t m = 0; m < count; ++m)
    if (hbad[m]) {
      P->sell_ok[m] = 0;
      P->dm[m].sell_ptr = nullptr;
      P->dm[m].sell_val = nullptr;
      P->dm[m].sell_off = nullptr;
      P->dm[m].sell_lo = nullptr;
    }
  return BSP_OK;
}

// The row-statistics choice: SELL-32 for every qualifying matrix (rows even
// enough that padding adds at most 1/8: every access coalesced and no
// row-pointer round trip, against CSR's per-row dependent loads).
int32_t model_format(const bsp_batch_plan P, int32_t m) { return P->sell_ok[m]; }
}  // namespace

extern "C" bsp_status bsp_batch_create(int32_t count, const bsp_batch_mat *mats, bsp_dtype dtype, int32_t nrhs,
                                       const bsp_batch_options *opt, bsp_batch_plan *out, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out && (count == 0 || mats) && count >= 0, "bad argument");
  BSP_CHECK_ARG(dtype == BSP_F64 || dtype == BSP_F32, "batched SpMV takes F64 or F32 values");
  BSP_CHECK_ARG(nrhs == 1 || nrhs == 8, "nrhs must be 1 or 8");
  *out = nullptr;
  bsp_batch_options o;
  bsp_batch_default_options(&o);
  if (opt) o = *opt;
  BSP_CHECK_ARG(o.seg_nnz >= 32 && o.long_row_nnz >= o.seg_nnz, "need 32 <= seg_nnz <= long_row_nnz");
  const size_t es = dtype == BSP_F64 ? 8 : 4;
  for (int32_t m = 0; m < count; ++m) {
    const bsp_batch_mat &A = mats[m];
    BSP_CHECK_ARG(A.rows >= 0 && A.cols >= 0 && A.nnz >= 0 && A.rowPtr, "bad matrix descriptor");
    BSP_CHECK_ARG(A.nnz == 0 || (A.colIdx && A.values), "bad matrix descriptor");
    BSP_CHECK_ARG(A.rows == 0 || A.y, "null y");
    BSP_CHECK_ARG(A.cols == 0 || A.x, "null x");
    if (nrhs == 8)
      BSP_CHECK_ARG((uintptr_t)A.x % 16 == 0 && (uintptr_t)A.y % 16 == 0, "8-RHS x / y must be 16-byte aligned");
    (void)es;
  }
  cudaStream_t s = as_stream(stream);
  bsp_batch_plan P = new bsp_batch_plan_s();
  P->count = count;
  P->nrhs = nrhs;
  P->dtype = dtype;
  P->opt = o;
  P->host_mats.assign(mats, mats + count);
  P->lens.resize(count);
  P->lanes.assign(count, 1);
  auto fail = [&](bsp_status st) {
    bsp_batch_destroy(P);
    return st;
  };
  // row lengths from the device row pointers
  std::vector<int32_t> rp;
  for (int32_t m = 0; m < count; ++m) {
    const bsp_batch_mat &A = mats[m];
    rp.resize((size_t)A.rows + 1);
    if (cudaMemcpyAsync(rp.data(), A.rowPtr, rp.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("bsp_batch_create: reading a row pointer failed");
      return fail(BSP_ERR_CUDA);
    }
    if (rp[0] != 0 || rp[A.rows] != A.nnz) {
      set_error("bsp_batch_create: rowPtr[0] must be 0 and rowPtr[rows] == nnz");
      return fail(BSP_ERR_INVALID);
    }
    auto &L = P->lens[m];
    L.resize(A.rows);
    for (int32_t r = 0; r < A.rows; ++r) L[r] = rp[r + 1] - rp[r];
    P->total_nnz += A.nnz;
    P->lanes[m] = model_lanes(L, o.long_row_nnz, nrhs);
  }
  P->dm.resize(count);
  for (int32_t m = 0; m < count; ++m)
    P->dm[m] = {mats[m].rowPtr, mats[m].colIdx, mats[m].values, mats[m].x, mats[m].y, mats[m].rows, mats[m].cols,
                nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  bsp_status st = build_sell(P, s);
  if (st != BSP_OK) return fail(st);
  P->fmt.assign(count, 0);
  for (int32_t m = 0; m < count; ++m) P->fmt[m] = model_format(P, m);
  if (dalloc(&P->d_mats, (size_t)count, s) != BSP_OK || dalloc(&P->d_next, (size_t)count + 1, s) != BSP_OK)
    return fail(BSP_ERR_ALLOC);
  if (count > 0 &&
      cudaMemcpyAsync(P->d_mats, P->dm.data(), P->dm.size() * sizeof(BatchMatDev), cudaMemcpyHostToDevice, s) !=
          cudaSuccess) {
    set_error("bsp_batch_create: copying descriptors failed");
    return fail(BSP_ERR_CUDA);
  }
  st = batch_build(P, s);
  if (st != BSP_OK) return fail(st);
  if (o.tune == 1) {
    // time every lane count on the matrices kept in CSR with one launch per
    // matrix and keep the fastest (outputs are overwritten, inputs
    // untouched).  The SELL-32 matrices stay SELL: timed the same way, one
    // matrix per launch, SELL lost to CSR on most banded matrices, yet the
    // batched launch with every qualifying matrix in SELL was the fastest
    // (512-matrix batch, FP64: 201.3 us against 213.9 with the per-matrix
    // choice and 227.7 all CSR).
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int cand[6] = {1, 2, 4, 8, 16, 32};
    std::vector<float> best(count, 1e30f);
    std::vector<int> best_l(P->lanes);
    for (int ci = 0; ci < 6 && st == BSP_OK; ++ci) {
      for (int32_t m = 0; m < count; ++m) P->lanes[m] = cand[ci];
      st = batch_build(P, s);
      for (int32_t m = 0; m < count && st == BSP_OK; ++m) {
        if (P->fmt[m] != 0) continue;
        float tmin = 1e30f;
        for (int rep = 0; rep < 3 && st == BSP_OK; ++rep) {
          cudaEventRecord(e0, s);
          st = batch_launch_one(P, m, s);
          cudaEventRecord(e1, s);
          cudaEventSynchronize(e1);
          float ms = 0;
          cudaEventElapsedTime(&ms, e0, e1);
          if (rep > 0) tmin = std::min(tmin, ms);
        }
        if (tmin < best[m]) {
          best[m] = tmin;
          best_l[m] = cand[ci];
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != BSP_OK) return fail(st);
    P->lanes = best_l;
    st = batch_build(P, s);
    if (st != BSP_OK) return fail(st);
  }
  st = capture(P);
  if (st != BSP_OK) return fail(st);
  *out = P;
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_run(bsp_batch_plan P, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P, "null plan");
  cudaStream_t s = as_stream(stream);
  if (P->graph) {
    BSP_CUDA(cudaGraphLaunch(P->graph, s));
    return BSP_OK;
  }
  BSP_CUDA(cudaMemsetAsync(P->d_next, 0, sizeof(int32_t), s));
  return dispatch(P, P->d_items, P->nitems, P->d_next, P->grid, s);
}

extern "C" bsp_status bsp_batch_run_separate(bsp_batch_plan P, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P, "null plan");
  cudaStream_t s = as_stream(stream);
  for (int32_t m = 0; m < P->count; ++m) BSP_TRY(batch_launch_one(P, m, s));
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_set_vectors(bsp_batch_plan P, int32_t m, const void *x, void *y,
                                            bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P && m >= 0 && m < P->count, "bad plan or matrix index");
  if (P->nrhs == 8) BSP_CHECK_ARG((uintptr_t)x % 16 == 0 && (uintptr_t)y % 16 == 0, "x / y must be 16-byte aligned");
  const bsp_batch_mat &A = P->host_mats[m];
  BSP_CHECK_ARG((A.cols == 0 || x) && (A.rows == 0 || y), "null vector");
  cudaStream_t s = as_stream(stream);
  P->host_mats[m].x = x;
  P->host_mats[m].y = y;
  P->dm[m].x = x;
  P->dm[m].y = y;
  const BatchMatDev d = P->dm[m];
  // the descriptor is read by the kernel: update it in stream order
  BSP_CUDA(cudaMemcpyAsync(P->d_mats + m, &d, sizeof(d), cudaMemcpyHostToDevice, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_lanes(bsp_batch_plan P, int32_t *lanes) {
  clear_error();
  BSP_CHECK_ARG(P && lanes, "null pointer");
  for (int32_t m = 0; m < P->count; ++m) lanes[m] = P->fmt[m] != 0 ? 0 : P->lanes[m];
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_formats(bsp_batch_plan P, int32_t *formats) {
  clear_error();
  BSP_CHECK_ARG(P && formats, "null pointer");
  for (int32_t m = 0; m < P->count; ++m) formats[m] = P->fmt[m];
  return BSP_OK;
}

extern "C" bsp_status bsp_batch_stats(bsp_batch_plan P, int64_t *items, int64_t *long_segments,
                                      int64_t *total_nnz) {
  clear_error();
  BSP_CHECK_ARG(P, "null plan");
  if (items) *items = P->nitems;
  if (long_segments) *long_segments = P->nseg;
  if (total_nnz) *total_nnz = P->total_nnz;
  return BSP_OK;
}
