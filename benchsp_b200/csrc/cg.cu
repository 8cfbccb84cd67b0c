// Conjugate gradients on the device: plain FP64 CG and mixed-precision CG
// with reliable updates.  The reference has no solver (the CG /
// mixed-precision rows are absent there); this is the precision form of the
// benchmark's CG configuration: 3-D 7-point Poisson, tolerance 1e-10 on
// ||b - A x|| / ||b|| checked in FP64.
//
// Mixed precision: the matrix is stored a second time, in SELL-32 layout
// (slices of 32 consecutive rows padded to the slice's longest row; entry k of
// the slice's row l at slice_off + 32 k + l, so the 32 rows of a warp read
// each k with one coalesced access), with values in FP32, FP16 or BF16.
// FP16/BF16 values carry one power-of-two exponent per row (v = stored * 2^e,
// the row's largest magnitude scaled into [1, 2); the row sum is scaled once),
// and column indices are stored as int16 offsets from the row
// when every |col - row| < 32768 (banded matrices), else int32.  FP16/BF16
// values with int16 offsets are packed into one 32-bit word per entry.  A
// nonzero then moves 4 bytes instead of 12 (FP64 + int32).  CG iterations
// run on that matrix with FP32 vectors (dot products in FP64).
// The FP64 state is the solution x64 and the true residual: whenever the
// iterated residual has dropped by `reliable_delta` since the last update,
// x64 += x32, r = b - A x64 is recomputed in FP64 with the FP64 matrix and
// replaces the iterated residual, and the search direction is kept (CG with
// reliable updates), so the iteration count stays close to plain FP64 CG while
// most bytes move at low precision.
//
// One CG iteration is two kernels:
//   A. beta = rr_k / rr_{k-1}; p_k = r_k + beta p_{k-1} formed on the fly for
//      every gathered column (r and p_{k-1} are read, p_k written for the own
//      row into the other p buffer); q = A p_k; partials of p_k.q;
//   B. alpha = rr_k / p.q; x += alpha p_k; r -= alpha q; partials of r.r.
// Every CTA reduces the previous kernel's per-CTA partials in the same order
// (deterministic, no atomics).  Scalars ping-pong between two slots by
// iteration parity so no CTA reads a value written in its own launch.  Zero
// denominators freeze the iteration (alpha = beta = 0), so iterations run
// after convergence inside a captured graph are harmless.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kCgThreads = 256;
constexpr int kRowFirst = 8;  // row entries loaded together per lane

template <typename V> __device__ __forceinline__ float lp_to_float(V v);
template <> __device__ __forceinline__ float lp_to_float<float>(float v) { return v; }
template <> __device__ __forceinline__ float lp_to_float<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float lp_to_float<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// 2^e as a float built from its exponent bits (|e| <= 126).
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }

// Deterministic block sum of one double per thread (fixed shuffle tree, then
// the warp totals in order).  Valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *smem /* [kCgThreads/32] */) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kCgThreads / 32; ++w) t += smem[w];
  __syncthreads();
  return t;
}

// Sum of n partials in index order; every CTA gets the same value.
__device__ __forceinline__ double reduce_partials(const double *__restrict__ part, int n, double *smem) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kCgThreads) s += __ldcg(part + i);
  s = block_sum(s, smem);
  __shared__ double bcast;
  if (threadIdx.x == 0) bcast = s;
  __syncthreads();
  return bcast;
}

// Matrix access: values V with optional group exponents, columns int32 or
// int16 offsets from the row.
// kPacked (FP16/BF16 values with int16 offsets): one 32-bit word per entry,
// value bits low, offset high, so one load gives both.
template <typename V, typename VT, bool SCALED, bool DELTA16>
struct CgMat {
  static constexpr bool kPacked = SCALED && DELTA16 && sizeof(V) == 2;
  const int32_t *rowPtr;  // CSR row pointers (FP64 mode)
  const void *cols;
  const V *val;           // SELL values, or the packed words when kPacked
  const int8_t *exps;
  const int32_t *slice_len;  // SELL-32 (mixed modes)
  const int64_t *slice_off;
  int32_t uniform_len;       // > 0: every slice has this length, offsets are sl * 32 * uniform_len
  __device__ __forceinline__ int64_t col(int64_t r, int32_t j) const {
    if (DELTA16) return r + (int64_t) reinterpret_cast<const int16_t *>(cols)[j];
    return reinterpret_cast<const int32_t *>(cols)[j];
  }
  __device__ __forceinline__ VT value(int32_t j) const { return (VT)val[j]; }  // CSR (FP64) path
};

// Kernel A: p_k = r + beta p_prev (own row stored, gathered columns formed on
// the fly), q = A p_k, partials of p_k.q.  rr_part = partials of rr_k;
// rr_prev_slot = rr_{k-1}; rr_slot receives rr_k (written by CTA 0).
// LPR (FP64 CSR path only): lanes per row; rows longer than ~10 entries
// get 2, 4 or 8 lanes that split the row's entries (4 loads in flight each)
// and combine by shuffle, instead of one thread walking the row.
// The FP64 CSR path fits 40 registers without spills: 6 resident CTAs per SM
// instead of 4 (Poisson 128^3 FP64 CG 37.0 -> 35.9 ms); so does the FP32
// SELL form with 32-bit columns (its default since the uniform-slice field).
// The other SELL forms keep the default (the same cap cost them 15%).
template <typename V, typename VT, bool SCALED, bool DELTA16, int LPR = 1>
__global__ void __launch_bounds__(kCgThreads, (sizeof(V) == 8 || (sizeof(V) == 4 && !DELTA16)) ? 6 : 0)
    cg_dir_spmv_kernel(int32_t n, CgMat<V, VT, SCALED, DELTA16> A,
                                                                 const VT *__restrict__ r,
                                                                 const VT *__restrict__ p_prev,
                                                                 VT *__restrict__ p, VT *__restrict__ q,
                                                                 const double *__restrict__ rr_part, int npart,
                                                                 const double *__restrict__ rr_prev_slot,
                                                                 double *__restrict__ rr_slot,
                                                                 double *__restrict__ pq_part) {
  __shared__ double smem[kCgThreads / 32];
  const double rr = reduce_partials(rr_part, npart, smem);
  const double rr_prev = *rr_prev_slot;
  const double beta = (rr_prev != 0.0 && isfinite(rr)) ? rr / rr_prev : 0.0;
  const VT bt = (VT)beta;
  double dot = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kCgThreads;
  if constexpr (sizeof(V) < 8 || DELTA16) {
    // SELL-32: warp = slice (the grid stride is a multiple of 32 rows); the
    // row's power-of-two scale is applied once to its sum; offsets are 32-bit
    // (the padded matrix has < 2^31 entries).  FP64 values (V = double, 16-bit
    // column offsets) are loaded and multiplied in FP64.
    using Mat = CgMat<V, VT, SCALED, DELTA16>;
    using AV = typename std::conditional<sizeof(V) == 8, double, float>::type;
    const int lane = threadIdx.x & 31;
    for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i - lane < n; i += stride) {
      const int32_t sl = (int32_t)(i >> 5);
      // uniform slices (16-bit offset forms; the 32-bit column form would
      // need 8 more registers): length and offset without loads
      const bool uni = DELTA16 && A.uniform_len > 0;
      const int32_t len = uni ? A.uniform_len : A.slice_len[sl];
      const uint32_t base = uni ? (uint32_t)sl * 32u * (uint32_t)A.uniform_len : (uint32_t)A.slice_off[sl];
      const uint32_t off = base + lane;
      const bool live = i < n;
      const int32_t row = (int32_t)i;
      VT acc = VT(0);
      const float row_scale = (SCALED && live) ? pow2f(A.exps[i]) : 1.f;
      {
        const int32_t kb = 0, kn = len;
        for (int32_t k0 = 0; k0 < kn; k0 += kRowFirst) {
          int32_t c[kRowFirst];
          AV a[kRowFirst];
#pragma unroll
          for (int k = 0; k < kRowFirst; ++k) {
            c[k] = row;
            a[k] = AV(0);
            if (k0 + k < kn) {
              const uint32_t j = off + (uint32_t)(kb + k0 + k) * 32u;
              if constexpr (Mat::kPacked) {
                const uint32_t w = __ldg(reinterpret_cast<const uint32_t *>(A.val) + j);
                const unsigned short vb = (unsigned short)(w & 0xffffu);
                if constexpr (std::is_same<V, __half>::value)
                  a[k] = __half2float(__ushort_as_half(vb));
                else
                  a[k] = __bfloat162float(__ushort_as_bfloat16(vb));
                c[k] = row + (int32_t)(int16_t)(w >> 16);
              } else {
                if constexpr (sizeof(V) == 8)
                  a[k] = __ldg(A.val + j);
                else
                  a[k] = lp_to_float<V>(__ldg(A.val + j));
                if (DELTA16)
                  c[k] = row + (int32_t)__ldg(reinterpret_cast<const int16_t *>(A.cols) + j);
                else
                  c[k] = __ldg(reinterpret_cast<const int32_t *>(A.cols) + j);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < kRowFirst; ++k)
            if (k0 + k < kn && live) acc = fma((VT)a[k], fma(bt, __ldg(p_prev + c[k]), __ldg(r + c[k])), acc);
        }
      }
      if constexpr (SCALED) acc *= row_scale;
      if (live) {
        const VT pi = fma(bt, p_prev[i], r[i]);
        p[i] = pi;
        q[i] = acc;
        dot += (double)acc * (double)pi;
      }
    }
  } else if constexpr (LPR > 1) {
    // warp-uniform loop: each pass covers 32 / LPR consecutive rows per warp
    const int lane = threadIdx.x & 31, sub = lane & (LPR - 1);
    const int64_t rstride = stride / LPR;
    for (int64_t base = ((int64_t)blockIdx.x * kCgThreads + (threadIdx.x & ~31)) / LPR; base < n; base += rstride) {
      const int64_t i = base + lane / LPR;
      const bool live = i < n;
      VT acc = VT(0);
      if (live) {
        const int32_t e = A.rowPtr[i + 1];
        int32_t j = A.rowPtr[i] + sub;
        for (; j + 3 * LPR < e; j += 4 * LPR) {
          int64_t c[4];
          VT a[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            c[k] = A.col(i, j + k * LPR);
            a[k] = A.value(j + k * LPR);
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) acc = fma(a[k], fma(bt, __ldg(p_prev + c[k]), __ldg(r + c[k])), acc);
        }
        for (; j < e; j += LPR) {
          const int64_t cj = A.col(i, j);
          acc = fma(A.value(j), fma(bt, __ldg(p_prev + cj), __ldg(r + cj)), acc);
        }
      }
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (live && sub == 0) {
        const VT pi = fma(bt, p_prev[i], r[i]);
        p[i] = pi;
        q[i] = acc;
        dot += (double)acc * (double)pi;
      }
    }
  } else
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += stride) {
    const int32_t s = A.rowPtr[i], e = A.rowPtr[i + 1];
    int64_t c[kRowFirst];
    VT a[kRowFirst];
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k) {
      const int32_t j = s + k;
      c[k] = j < e ? A.col(i, j) : -1;
      a[k] = j < e ? A.value(j) : VT(0);
    }
    VT acc = VT(0);
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k)
      if (c[k] >= 0) acc = fma(a[k], fma(bt, __ldg(p_prev + c[k]), __ldg(r + c[k])), acc);
    for (int32_t j = s + kRowFirst; j < e; ++j) {
      const int64_t cj = A.col(i, j);
      acc = fma(A.value(j), fma(bt, __ldg(p_prev + cj), __ldg(r + cj)), acc);
    }
    const VT pi = fma(bt, p_prev[i], r[i]);
    p[i] = pi;
    q[i] = acc;
    dot += (double)acc * (double)pi;
  }
  const double t = block_sum(dot, smem);
  if (threadIdx.x == 0) {
    pq_part[blockIdx.x] = t;
    if (blockIdx.x == 0) *rr_slot = rr;
  }
}

// Kernel B: alpha = rr_k / p.q; x += alpha p; r -= alpha q; partials of r.r.
// 16-byte vector accesses (4 floats or 2 doubles per load), two in flight
// per thread; the scalar tail covers n not divisible by the vector width.
template <typename VT> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int W = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int W = 2; };

__device__ __forceinline__ float vget(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
__device__ __forceinline__ double vget(const double2 &v, int k) { return k == 0 ? v.x : v.y; }
__device__ __forceinline__ void vset(float4 &v, int k, float a) {
  if (k == 0) v.x = a; else if (k == 1) v.y = a; else if (k == 2) v.z = a; else v.w = a;
}
__device__ __forceinline__ void vset(double2 &v, int k, double a) {
  if (k == 0) v.x = a; else v.y = a;
}

template <typename VT>
__global__ void __launch_bounds__(kCgThreads) cg_update_kernel(int32_t n, const double *__restrict__ pq_part,
                                                               int npart, const double *__restrict__ rr_slot,
                                                               VT *__restrict__ x, VT *__restrict__ r,
                                                               const VT *__restrict__ p, const VT *__restrict__ q,
                                                               double *__restrict__ rr_part) {
  using V = typename Vec16<VT>::T;
  constexpr int W = Vec16<VT>::W;
  constexpr int U = 2;
  __shared__ double smem[kCgThreads / 32];
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * kCgThreads;
  V *xv = reinterpret_cast<V *>(x);
  V *rv = reinterpret_cast<V *>(r);
  const V *pv = reinterpret_cast<const V *>(p);
  const V *qv = reinterpret_cast<const V *>(q);
  V P[U], Q[U], X[U], R[U];
  auto load = [&](int64_t i0) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < nv) {
        P[u] = pv[i];
        Q[u] = qv[i];
        X[u] = xv[i];
        R[u] = rv[i];
      }
    }
  };
  // the first pass's vectors do not depend on alpha: their loads are in
  // flight while the CTA sums the p.q partials
  const int64_t first = (int64_t)blockIdx.x * kCgThreads + threadIdx.x;
  load(first);
  const double pq = reduce_partials(pq_part, npart, smem);
  const double rr = *rr_slot;
  const double alpha = (pq != 0.0 && rr != 0.0 && isfinite(pq)) ? rr / pq : 0.0;
  const VT a = (VT)alpha;
  double s = 0.0;
  for (int64_t i0 = first; i0 < nv; i0 += U * stride) {
    if (i0 != first) load(i0);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < nv) {
#pragma unroll
        for (int k = 0; k < W; ++k) {
          vset(X[u], k, fma(a, vget(P[u], k), vget(X[u], k)));
          const VT ri = fma(-a, vget(Q[u], k), vget(R[u], k));
          vset(R[u], k, ri);
          s += (double)ri * (double)ri;
        }
        xv[i] = X[u];
        rv[i] = R[u];
      }
    }
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += stride) {
    x[i] = fma(a, p[i], x[i]);
    const VT ri = fma(-a, q[i], r[i]);
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  const double t = block_sum(s, smem);
  if (threadIdx.x == 0) rr_part[blockIdx.x] = t;
}

// ---------------------------------------------------------------------------
// Preconditioned CG (Jacobi: BS = 1; block-Jacobi: BS = 4 or 8 consecutive
// rows).  M^{-1} is stored in the iteration precision: dinv[n] for BS = 1,
// else the inverted diagonal blocks, BS*BS row-major per block (the last block
// padded with identity rows).  The preconditioned iteration keeps the two
// kernels: kernel A gathers z = M^{-1} r where it gathered r and reduces the
// r.z partials where it reduced r.r; the update kernel below also applies
// M^{-1} to the new residual and writes both the r.r partials (convergence
// checks) and the r.z partials (the next direction).
//
// One thread per group of G rows, G = 8 for 8x8 blocks and 4 otherwise (BS
// divides G, so blocks never straddle groups; 4 rows keep the FP64 kernel
// near 60 registers, 8 rows of five vectors needed 100 and halved the
// resident warps): 16-byte vector accesses for full groups, bounds-checked
// scalars for the last partial group.
template <int BS> struct PrecGroup { static constexpr int G = BS == 8 ? 8 : 4; };

template <typename VT, int G>
__device__ __forceinline__ void ldg_rows(const VT *__restrict__ p, VT (&v)[G]) {
  using V = typename Vec16<VT>::T;
  constexpr int W = Vec16<VT>::W;
  const V *pv = reinterpret_cast<const V *>(p);
#pragma unroll
  for (int u = 0; u < G / W; ++u) {
    const V t = pv[u];
#pragma unroll
    for (int k = 0; k < W; ++k) v[u * W + k] = vget(t, k);
  }
}

template <typename VT, int G>
__device__ __forceinline__ void stg_rows(VT *__restrict__ p, const VT (&v)[G]) {
  using V = typename Vec16<VT>::T;
  constexpr int W = Vec16<VT>::W;
  V *pv = reinterpret_cast<V *>(p);
#pragma unroll
  for (int u = 0; u < G / W; ++u) {
    V t;
#pragma unroll
    for (int k = 0; k < W; ++k) vset(t, k, v[u * W + k]);
    pv[u] = t;
  }
}

// z = M^{-1} r for the G-row group starting at row i0 (rows >= n hold r = 0).
template <typename VT, int BS, int G>
__device__ __forceinline__ void apply_minv(const VT *__restrict__ minv, int64_t i0, int32_t n, const VT (&r)[G],
                                           VT (&z)[G]) {
  if constexpr (BS == 1) {
    if (i0 + G <= n) {
      VT d[G];
      ldg_rows<VT, G>(minv + i0, d);
#pragma unroll
      for (int k = 0; k < G; ++k) z[k] = d[k] * r[k];
    } else {
#pragma unroll
      for (int k = 0; k < G; ++k) z[k] = i0 + k < n ? minv[i0 + k] * r[k] : VT(0);
    }
  } else {
    const int64_t nb = ((int64_t)n + BS - 1) / BS;
#pragma unroll
    for (int b = 0; b < G / BS; ++b) {
      const int64_t blk = i0 / BS + b;
      if (blk >= nb) {
#pragma unroll
        for (int i = 0; i < BS; ++i) z[b * BS + i] = VT(0);
        continue;
      }
      const VT *Mb = minv + blk * BS * BS;
#pragma unroll
      for (int i = 0; i < BS; ++i) {
        VT row[BS];
        ldg_rows<VT, BS>(Mb + i * BS, row);
        VT acc = VT(0);
#pragma unroll
        for (int j = 0; j < BS; ++j) acc = fma(row[j], r[b * BS + j], acc);
        z[b * BS + i] = acc;
      }
    }
  }
}

// UPDATE: alpha = rz / p.q; x += alpha p; r -= alpha q; then z = M^{-1} r,
// partials of r.r and r.z.  !UPDATE: z = M^{-1} r and r.z partials only
// (after the residual was replaced).
template <typename VT, int BS, bool UPDATE>
__global__ void __launch_bounds__(kCgThreads, 4) cg_update_prec_kernel(int32_t n, const double *__restrict__ pq_part,
                                                                    int npart, const double *__restrict__ rz_slot,
                                                                    VT *__restrict__ x, VT *__restrict__ r,
                                                                    VT *__restrict__ z, const VT *__restrict__ p,
                                                                    const VT *__restrict__ q,
                                                                    const VT *__restrict__ minv,
                                                                    double *__restrict__ rr_part,
                                                                    double *__restrict__ rz_part) {
  __shared__ double smem[kCgThreads / 32];
  VT a = VT(0);
  if constexpr (UPDATE) {
    const double pq = reduce_partials(pq_part, npart, smem);
    const double rz = *rz_slot;
    const double alpha = (pq != 0.0 && rz != 0.0 && isfinite(pq)) ? rz / pq : 0.0;
    a = (VT)alpha;
  }
  constexpr int G = PrecGroup<BS>::G;
  double srr = 0.0, srz = 0.0;
  const int64_t ng = ((int64_t)n + G - 1) / G;
  const int64_t stride = (int64_t)gridDim.x * kCgThreads;
  for (int64_t g = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; g < ng; g += stride) {
    const int64_t i0 = g * G;
    const bool full = i0 + G <= n;
    VT R[G], Z[G];
    if (full) {
      ldg_rows<VT, G>(r + i0, R);
    } else {
#pragma unroll
      for (int k = 0; k < G; ++k) R[k] = i0 + k < n ? r[i0 + k] : VT(0);
    }
    if constexpr (UPDATE) {
      VT P[G], Q[G], X[G];
      if (full) {
        ldg_rows<VT, G>(p + i0, P);
        ldg_rows<VT, G>(q + i0, Q);
        ldg_rows<VT, G>(x + i0, X);
      } else {
#pragma unroll
        for (int k = 0; k < G; ++k) {
          const bool in = i0 + k < n;
          P[k] = in ? p[i0 + k] : VT(0);
          Q[k] = in ? q[i0 + k] : VT(0);
          X[k] = in ? x[i0 + k] : VT(0);
        }
      }
#pragma unroll
      for (int k = 0; k < G; ++k) {
        X[k] = fma(a, P[k], X[k]);
        R[k] = fma(-a, Q[k], R[k]);
        srr += (double)R[k] * (double)R[k];
      }
      if (full) {
        stg_rows<VT, G>(x + i0, X);
        stg_rows<VT, G>(r + i0, R);
      } else {
#pragma unroll
        for (int k = 0; k < G; ++k)
          if (i0 + k < n) {
            x[i0 + k] = X[k];
            r[i0 + k] = R[k];
          }
      }
    }
    apply_minv<VT, BS, G>(minv, i0, n, R, Z);
#pragma unroll
    for (int k = 0; k < G; ++k) srz += (double)R[k] * (double)Z[k];
    if (full) {
      stg_rows<VT, G>(z + i0, Z);
    } else {
#pragma unroll
      for (int k = 0; k < G; ++k)
        if (i0 + k < n) z[i0 + k] = Z[k];
    }
  }
  if constexpr (UPDATE) {
    const double t = block_sum(srr, smem);
    if (threadIdx.x == 0) rr_part[blockIdx.x] = t;
  }
  const double t2 = block_sum(srz, smem);
  if (threadIdx.x == 0) rz_part[blockIdx.x] = t2;
}

// M^{-1} from the CSR matrix: thread per block of BS rows; the block's
// entries (columns in the block's own range, found by binary search in the
// sorted row, duplicates summed) inverted by Gauss-Jordan elimination with
// partial pivoting in FP64.  A zero or non-finite pivot sets *bad.
template <typename VT, int BS>
__global__ void cg_minv_kernel(int32_t n, const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
                               const double *__restrict__ val, VT *__restrict__ minv, int32_t *__restrict__ bad) {
  const int64_t nb = ((int64_t)n + BS - 1) / BS;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
    double M[BS][BS], I[BS][BS];
    const int64_t lo = b * BS;
    for (int i = 0; i < BS; ++i)
      for (int j = 0; j < BS; ++j) {
        M[i][j] = 0.0;
        I[i][j] = i == j ? 1.0 : 0.0;
      }
    for (int i = 0; i < BS; ++i) {
      const int64_t row = lo + i;
      if (row >= n) {
        M[i][i] = 1.0;  // padding of the last block
        continue;
      }
      int32_t s = rowPtr[row], e = rowPtr[row + 1];
      while (s < e) {  // first column >= lo
        const int32_t m = s + ((e - s) >> 1);
        if (colIdx[m] < lo)
          s = m + 1;
        else
          e = m;
      }
      for (int32_t j = s; j < rowPtr[row + 1] && colIdx[j] < lo + BS; ++j) M[i][colIdx[j] - lo] += val[j];
    }
    bool ok = true;
    for (int c = 0; c < BS && ok; ++c) {
      int piv = c;
      for (int i = c + 1; i < BS; ++i)
        if (fabs(M[i][c]) > fabs(M[piv][c])) piv = i;
      if (!(fabs(M[piv][c]) > 0.0) || !isfinite(M[piv][c])) {
        ok = false;
        break;
      }
      if (piv != c)
        for (int j = 0; j < BS; ++j) {
          double t = M[c][j];
          M[c][j] = M[piv][j];
          M[piv][j] = t;
          t = I[c][j];
          I[c][j] = I[piv][j];
          I[piv][j] = t;
        }
      const double inv = 1.0 / M[c][c];
      for (int j = 0; j < BS; ++j) {
        M[c][j] *= inv;
        I[c][j] *= inv;
      }
      for (int i = 0; i < BS; ++i)
        if (i != c) {
          const double f = M[i][c];
          if (f != 0.0)
            for (int j = 0; j < BS; ++j) {
              M[i][j] -= f * M[c][j];
              I[i][j] -= f * I[c][j];
            }
        }
    }
    if (!ok) atomicExch(bad, 1);
    for (int i = 0; i < BS; ++i)
      for (int j = 0; j < BS; ++j) minv[b * BS * BS + i * BS + j] = (VT)(ok ? I[i][j] : (i == j ? 1.0 : 0.0));
  }
}

// FP64 true residual r = b - A x, partials of ||r||^2; optionally also the
// inner-precision copy r_lp = (VT) r and its partials (reliable update), and
// the partials of ||r - r_lp_old||^2, the distance of the true residual from
// the iterated one it replaces (part_dev, may be null).
template <typename VT>
__global__ void __launch_bounds__(kCgThreads) cg_residual_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                                 const int32_t *__restrict__ colIdx,
                                                                 const double *__restrict__ val,
                                                                 const double *__restrict__ b,
                                                                 const double *__restrict__ x,
                                                                 double *__restrict__ r, VT *__restrict__ r_lp,
                                                                 double *__restrict__ part,
                                                                 double *__restrict__ part_lp,
                                                                 double *__restrict__ part_dev = nullptr) {
  __shared__ double smem[kCgThreads / 32];
  double nrm = 0.0, nrm_lp = 0.0, dev = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kCgThreads;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += stride) {
    const int32_t s = rowPtr[i], e = rowPtr[i + 1];
    int32_t c[kRowFirst];
    double a[kRowFirst];
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k) {
      c[k] = s + k < e ? colIdx[s + k] : -1;
      a[k] = s + k < e ? val[s + k] : 0.0;
    }
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k)
      if (c[k] >= 0) acc = fma(a[k], __ldg(x + c[k]), acc);
    for (int32_t j = s + kRowFirst; j < e; ++j) acc = fma(val[j], __ldg(x + colIdx[j]), acc);
    const double ri = b[i] - acc;
    if (r) r[i] = ri;
    nrm += ri * ri;
    if (r_lp) {
      if (part_dev) {
        const double d = ri - (double)r_lp[i];
        dev += d * d;
      }
      const VT v = (VT)ri;
      r_lp[i] = v;
      nrm_lp += (double)v * (double)v;
    }
  }
  double t = block_sum(nrm, smem);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  if (r_lp) {
    t = block_sum(nrm_lp, smem);
    if (threadIdx.x == 0) part_lp[blockIdx.x] = t;
  }
  if (part_dev) {
    t = block_sum(dev, smem);
    if (threadIdx.x == 0) part_dev[blockIdx.x] = t;
  }
}

// x64 += x_lp; x_lp = 0 (reliable update of the solution).
template <typename VT>
__global__ void cg_fold_kernel(int32_t n, VT *__restrict__ x_lp, double *__restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] += (double)x_lp[i];
    x_lp[i] = VT(0);
  }
}

// ---------------------------------------------------------------------------
// Flexible outer iteration for the mixed modes (FCG(1), one previous
// direction): the inner low-precision (P)CG, run until its residual has
// dropped by reliable_delta, is the preconditioner z = B(r) of an FP64 CG on
// the FP64 matrix.  Because B changes from step to step (and the inner matrix
// is only an approximation of A), the new direction is A-orthogonalised
// against the previous one explicitly: p = z - (z.q_prev / p_prev.q_prev) p_prev,
// q = A p, alpha = p.r / p.q.  Unlike residual replacement, the outer Krylov
// step keeps converging when the low-precision matrix is far from A.
//
// F1: z = (double) x_lp; x_lp = 0; partials of z.q_prev.
__global__ void __launch_bounds__(kCgThreads) fcg_z_kernel(int32_t n, float *__restrict__ x_lp,
                                                           double *__restrict__ z, const double *__restrict__ q_prev,
                                                           double *__restrict__ part) {
  __shared__ double smem[kCgThreads / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    const double zi = (double)x_lp[i];
    x_lp[i] = 0.f;
    z[i] = zi;
    s += zi * q_prev[i];
  }
  const double t = block_sum(s, smem);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// F2: p = z - gamma p_prev, gamma = z.q_prev / pq_prev (0 on the first step).
__global__ void __launch_bounds__(kCgThreads) fcg_dir_kernel(int32_t n, const double *__restrict__ part, int npart,
                                                             const double *__restrict__ pq_prev_slot,
                                                             const double *__restrict__ z, double *__restrict__ p) {
  __shared__ double smem[kCgThreads / 32];
  const double zq = reduce_partials(part, npart, smem);
  const double pq_prev = *pq_prev_slot;
  const double gamma = (pq_prev != 0.0 && isfinite(zq)) ? zq / pq_prev : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads)
    p[i] = gamma != 0.0 ? fma(-gamma, p[i], z[i]) : z[i];
}

// F3: q = A p (FP64 CSR); partials of p.q and p.r.
__global__ void __launch_bounds__(kCgThreads) fcg_spmv_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                              const int32_t *__restrict__ colIdx,
                                                              const double *__restrict__ val,
                                                              const double *__restrict__ p, double *__restrict__ q,
                                                              const double *__restrict__ r,
                                                              double *__restrict__ part_pq,
                                                              double *__restrict__ part_pr) {
  __shared__ double smem[kCgThreads / 32];
  double spq = 0.0, spr = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    const int32_t s0 = rowPtr[i], e0 = rowPtr[i + 1];
    int32_t c[kRowFirst];
    double a[kRowFirst];
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k) {
      c[k] = s0 + k < e0 ? colIdx[s0 + k] : -1;
      a[k] = s0 + k < e0 ? val[s0 + k] : 0.0;
    }
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kRowFirst; ++k)
      if (c[k] >= 0) acc = fma(a[k], __ldg(p + c[k]), acc);
    for (int32_t j = s0 + kRowFirst; j < e0; ++j) acc = fma(val[j], __ldg(p + colIdx[j]), acc);
    q[i] = acc;
    spq += p[i] * acc;
    spr += p[i] * r[i];
  }
  double t = block_sum(spq, smem);
  if (threadIdx.x == 0) part_pq[blockIdx.x] = t;
  t = block_sum(spr, smem);
  if (threadIdx.x == 0) part_pr[blockIdx.x] = t;
}

// F4: alpha = p.r / p.q; x += alpha p; r -= alpha q; r_lp = (float) r;
// partials of r.r and r_lp.r_lp; p.q kept in *pq_slot for the next F2.
__global__ void __launch_bounds__(kCgThreads) fcg_update_kernel(int32_t n, const double *__restrict__ part_pq,
                                                                const double *__restrict__ part_pr, int npart,
                                                                double *__restrict__ pq_slot,
                                                                double *__restrict__ x, double *__restrict__ r,
                                                                const double *__restrict__ p,
                                                                const double *__restrict__ q,
                                                                float *__restrict__ r_lp,
                                                                double *__restrict__ part_rr,
                                                                double *__restrict__ part_rr_lp) {
  __shared__ double smem[kCgThreads / 32];
  const double pq = reduce_partials(part_pq, npart, smem);
  const double pr = reduce_partials(part_pr, npart, smem);
  const double alpha = (pq > 0.0 && isfinite(pq) && isfinite(pr)) ? pr / pq : 0.0;
  double s = 0.0, sl = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    const float rl = (float)ri;
    r_lp[i] = rl;
    s += ri * ri;
    sl += (double)rl * (double)rl;
  }
  double t = block_sum(s, smem);
  if (threadIdx.x == 0) part_rr[blockIdx.x] = t;
  t = block_sum(sl, smem);
  if (threadIdx.x == 0) {
    part_rr_lp[blockIdx.x] = t;
    if (blockIdx.x == 0) *pq_slot = (pq > 0.0 && isfinite(pq)) ? pq : 0.0;
  }
}

__global__ void sum_partials_kernel(const double *__restrict__ part, int npart, double *__restrict__ out) {
  __shared__ double smem[kCgThreads / 32];
  const double s = reduce_partials(part, npart, smem);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Low-precision SELL-32 copy of the matrix.
__global__ void sell_len_kernel(int32_t n, const int32_t *__restrict__ rowPtr, int32_t *__restrict__ slice_len) {
  const int64_t ns = ((int64_t)n + 31) / 32;
  for (int64_t sl = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; sl < ns; sl += (int64_t)gridDim.x * blockDim.x) {
    int32_t m = 0;
    for (int64_t r = sl * 32; r < n && r < sl * 32 + 32; ++r) m = max(m, rowPtr[r + 1] - rowPtr[r]);
    slice_len[sl] = m;
  }
}

// One power-of-two exponent per row: the row's largest magnitude scaled into [1, 2).
__global__ void row_exp_kernel(int32_t n, const int32_t *__restrict__ rowPtr, const double *__restrict__ val,
                               int8_t *__restrict__ exps) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    double m = 0.0;
    for (int32_t j = rowPtr[r]; j < rowPtr[r + 1]; ++j) m = fmax(m, fabs(val[j]));
    int e = 0;
    if (m > 0.0) {
      frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
      e -= 1;
    }
    exps[r] = (int8_t)(e < -100 ? -100 : (e > 100 ? 100 : e));
  }
}

template <typename V>
__device__ __forceinline__ V from_float_lp(float f);
template <> __device__ __forceinline__ float from_float_lp<float>(float f) { return f; }
template <> __device__ __forceinline__ __half from_float_lp<__half>(float f) { return __float2half_rn(f); }
template <> __device__ __forceinline__ __nv_bfloat16 from_float_lp<__nv_bfloat16>(float f) { return __float2bfloat16_rn(f); }

// Thread per (slice row): its entries (scaled, converted) and columns (int16
// offsets or int32) into the slice; padding = value 0, column = the row
// itself (rows past n in the last slice: column 0, never gathered).
template <typename V, bool SCALED, bool D16, bool PACKED>
__global__ void sell_fill_kernel(int32_t n, const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
                                 const double *__restrict__ val, const int32_t *__restrict__ slice_len,
                                 const int64_t *__restrict__ slice_off, const int8_t *__restrict__ exps,
                                 V *__restrict__ out, void *__restrict__ cols) {
  const int64_t ns = ((int64_t)n + 31) / 32;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ns * 32; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sl = t >> 5, lane = t & 31;
    const int64_t self = t < n ? t : 0;
    const int32_t s0 = t < n ? rowPtr[t] : 0, e0 = t < n ? rowPtr[t + 1] : 0;
    for (int32_t k = 0; k < slice_len[sl]; ++k) {
      const int64_t j = slice_off[sl] + (int64_t)k * 32 + lane;
      double v = 0.0;
      int64_t c = self;
      if (s0 + k < e0) {
        v = val[s0 + k];
        c = colIdx[s0 + k];
        if (SCALED) v = ldexp(v, -(int)exps[t]);
      }
      V lv;
      if constexpr (sizeof(V) == 8)
        lv = v;  // the FP64 copy keeps the values exactly
      else
        lv = from_float_lp<V>((float)v);
      const int64_t d = c - self;
      if (PACKED) {
        unsigned short vb;
        memcpy(&vb, &lv, sizeof(vb));
        reinterpret_cast<uint32_t *>(out)[j] = (uint32_t)vb | ((uint32_t)(uint16_t)(int16_t)d << 16);
      } else {
        out[j] = lv;
        if (D16)
          reinterpret_cast<int16_t *>(cols)[j] = (int16_t)d;
        else
          reinterpret_cast<int32_t *>(cols)[j] = (int32_t)c;
      }
    }
  }
}

__global__ void cg_delta_check_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                      const int32_t *__restrict__ colIdx, int32_t *__restrict__ bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; ++j) {
      const int64_t d = (int64_t)colIdx[j] - i;
      if (d < -32768 || d > 32767) {
        atomicExch(bad, 1);
        break;
      }
    }
}

__global__ void f64_to_f32_kernel(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}


}  // namespace bsp

// ---------------------------------------------------------------------------
struct bsp_cg_plan_s {
  int32_t n = 0, nnz = 0;
  bsp_cg_options opt{};
  const int32_t *rowPtr = nullptr, *colIdx = nullptr;
  const double *val = nullptr;
  // low-precision copy of the matrix (mixed modes)
  void *lp_val = nullptr;
  int8_t *exps = nullptr;
  void *lp_cols = nullptr;     // int16 offsets or int32 columns (unpacked SELL)
  int32_t *slice_len = nullptr;
  int64_t *slice_off = nullptr;
  int32_t sell_uniform = 0;    // > 0: all slices padded to this length
  bool delta16 = false;
  bool sell64 = false;         // FP64 mode iterates on an FP64 SELL-32 copy
  // FP64 state
  double *x64 = nullptr, *r64 = nullptr;
  // iteration vectors: FP64 (mode FP64) or FP32 (mixed); p ping-pongs
  void *x = nullptr, *r = nullptr, *p[2] = {nullptr, nullptr}, *q = nullptr;
  double *part_pq = nullptr, *part_rr = nullptr, *part_res = nullptr;
  // preconditioning: prec_bs = 0 (none), 1 (Jacobi), 4 or 8 (block-Jacobi)
  int prec_bs = 0;
  int lpr = 1;  // FP64 mode: lanes per row of the direction/SpMV kernel
  void *z = nullptr, *minv = nullptr;
  double *part_rz = nullptr;
  // flexible outer iteration (mixed modes): FP64 p, q, z; r64 holds the
  // FP64 residual; partials of z.q_prev and p.r
  double *p64 = nullptr, *q64 = nullptr, *z64 = nullptr;
  double *part_zq = nullptr, *part_pr = nullptr;
  int64_t bytes_outer = 0;
  double *sc = nullptr, *h_sc = nullptr;  // [0],[1] rr slots, [2] ||b-Ax||^2, [3] ||b||^2, [4] rr after a chunk
  int grid = 0;    // update, residual and reduction kernels (writers of the rr partials)
  int grid_a = 0;  // direction/SpMV kernel (writer of the p.q partials)
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  int64_t bytes_iter = 0, bytes_residual = 0;
};

namespace bsp {

constexpr int kCgMaxCtasPerSm = 2048 / kCgThreads;
// Mixed modes: a replaced (true) residual whose distance from the iterated
// one exceeds kCgDeviation x its norm, or an iterated residual above kCgGrowth
// x the last true one, marks the low-precision matrix as too far from A for
// residual replacement (AUTO then switches to the flexible outer iteration).
// Measured: <= 0.006 where replacement keeps the FP64 iteration count, >= 0.13
// where it costs 1.5x-30x more iterations.
constexpr double kCgDeviation = 0.1;
constexpr double kCgGrowth = 1e4;
// Mixed modes: this many residual replacements in a row without a new lowest
// true residual end the solve (BSP_ERR_NOT_CONVERGED).
constexpr int kCgNoProgress = 6;
// Mixed modes: this many chunks without the inner drop force a residual
// replacement / outer step (an inner iteration that stagnates).
constexpr int kCgInnerChunks = 32;

// Resident CTAs per SM of the direction/SpMV kernel (a) and of the update
// kernel (b).
template <typename V, typename VT, bool SC, bool D16>
static void cg_occupancy(int &a, int &b) {
  a = b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, cg_dir_spmv_kernel<V, VT, SC, D16>, kCgThreads, 0) !=
      cudaSuccess)
    a = 4;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, cg_update_kernel<VT>, kCgThreads, 0) != cudaSuccess) b = 4;
  a = a < 1 ? 1 : (a > kCgMaxCtasPerSm ? kCgMaxCtasPerSm : a);
  b = b < 1 ? 1 : (b > kCgMaxCtasPerSm ? kCgMaxCtasPerSm : b);
}

// One resident wave (grid-stride loops inside).
static int cg_grid(int32_t n, int occ) {
  int64_t g = ceil_div(n, kCgThreads);
  const int64_t cap = (int64_t)sm_count() * occ;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

static bool cg_mixed(const bsp_cg_plan_s *P) { return P->opt.mode != BSP_CG_FP64; }

static void cg_plan_occupancy(const bsp_cg_plan_s *P, int &a, int &b) {
  const bool d = P->delta16;
  switch (P->opt.mode) {
    case BSP_CG_FP64:
      return P->sell64 ? cg_occupancy<double, double, false, true>(a, b)
                       : cg_occupancy<double, double, false, false>(a, b);
    case BSP_CG_MIXED_F32:
      return d ? cg_occupancy<float, float, false, true>(a, b) : cg_occupancy<float, float, false, false>(a, b);
    case BSP_CG_MIXED_F16:
      return d ? cg_occupancy<__half, float, true, true>(a, b) : cg_occupancy<__half, float, true, false>(a, b);
    default:
      return d ? cg_occupancy<__nv_bfloat16, float, true, true>(a, b)
               : cg_occupancy<__nv_bfloat16, float, true, false>(a, b);
  }
}

template <typename V, typename VT, bool SC, bool D16, int LPR = 1>
static void launch_iter(bsp_cg_plan_s *P, int k, cudaStream_t s) {
  constexpr bool csr = sizeof(V) == 8 && !D16;  // FP64 CSR; the other forms read the SELL copy
  CgMat<V, VT, SC, D16> A{P->rowPtr, csr ? (const void *)P->colIdx : (const void *)P->lp_cols,
                           (const V *)(csr ? (const void *)P->val : P->lp_val), P->exps,
                           P->slice_len, P->slice_off, P->sell_uniform};
  VT *r = (VT *)P->r, *x = (VT *)P->x, *q = (VT *)P->q;
  VT *pp = (VT *)P->p[k & 1], *pn = (VT *)P->p[(k + 1) & 1];
  const int g = P->grid, ga = P->grid_a;
  if (P->prec_bs == 0) {
    cg_dir_spmv_kernel<V, VT, SC, D16, LPR><<<ga, kCgThreads, 0, s>>>(P->n, A, r, pp, pn, q, P->part_rr, g,
                                                                  P->sc + ((k + 1) & 1), P->sc + (k & 1),
                                                                  P->part_pq);
    cg_update_kernel<VT><<<g, kCgThreads, 0, s>>>(P->n, P->part_pq, ga, P->sc + (k & 1), x, r, pn, q, P->part_rr);
    return;
  }
  // preconditioned: directions from z, r.z in the scalar slots
  VT *z = (VT *)P->z;
  const VT *mi = (const VT *)P->minv;
  cg_dir_spmv_kernel<V, VT, SC, D16, LPR><<<ga, kCgThreads, 0, s>>>(P->n, A, z, pp, pn, q, P->part_rz, g,
                                                                P->sc + ((k + 1) & 1), P->sc + (k & 1),
                                                                P->part_pq);
  const double *sl = P->sc + (k & 1);
  switch (P->prec_bs) {
    case 1:
      cg_update_prec_kernel<VT, 1, true><<<g, kCgThreads, 0, s>>>(P->n, P->part_pq, ga, sl, x, r, z, pn, q, mi,
                                                                   P->part_rr, P->part_rz);
      break;
    case 4:
      cg_update_prec_kernel<VT, 4, true><<<g, kCgThreads, 0, s>>>(P->n, P->part_pq, ga, sl, x, r, z, pn, q, mi,
                                                                   P->part_rr, P->part_rz);
      break;
    default:
      cg_update_prec_kernel<VT, 8, true><<<g, kCgThreads, 0, s>>>(P->n, P->part_pq, ga, sl, x, r, z, pn, q, mi,
                                                                   P->part_rr, P->part_rz);
  }
}

// z = M^{-1} r and the r.z partials, after the residual was replaced.
template <typename VT>
static void launch_prec(bsp_cg_plan_s *P, cudaStream_t s) {
  VT *r = (VT *)P->r, *z = (VT *)P->z;
  const VT *mi = (const VT *)P->minv;
  const int g = P->grid;
  switch (P->prec_bs) {
    case 1:
      cg_update_prec_kernel<VT, 1, false><<<g, kCgThreads, 0, s>>>(P->n, nullptr, 0, nullptr, nullptr, r, z, nullptr,
                                                                    nullptr, mi, nullptr, P->part_rz);
      break;
    case 4:
      cg_update_prec_kernel<VT, 4, false><<<g, kCgThreads, 0, s>>>(P->n, nullptr, 0, nullptr, nullptr, r, z, nullptr,
                                                                    nullptr, mi, nullptr, P->part_rz);
      break;
    default:
      cg_update_prec_kernel<VT, 8, false><<<g, kCgThreads, 0, s>>>(P->n, nullptr, 0, nullptr, nullptr, r, z, nullptr,
                                                                    nullptr, mi, nullptr, P->part_rz);
  }
}

static bsp_status cg_iteration(bsp_cg_plan_s *P, int k, cudaStream_t s) {
  if (P->sell64) {
    launch_iter<double, double, false, true>(P, k, s);
  } else if (!cg_mixed(P)) {
    switch (P->lpr) {
      case 2: launch_iter<double, double, false, false, 2>(P, k, s); break;
      case 4: launch_iter<double, double, false, false, 4>(P, k, s); break;
      case 8: launch_iter<double, double, false, false, 8>(P, k, s); break;
      default: launch_iter<double, double, false, false, 1>(P, k, s);
    }
  } else {
    const bool d = P->delta16;
    switch (P->opt.mode) {
      case BSP_CG_MIXED_F32:
        d ? launch_iter<float, float, false, true>(P, k, s) : launch_iter<float, float, false, false>(P, k, s);
        break;
      case BSP_CG_MIXED_F16:
        d ? launch_iter<__half, float, true, true>(P, k, s) : launch_iter<__half, float, true, false>(P, k, s);
        break;
      default:
        d ? launch_iter<__nv_bfloat16, float, true, true>(P, k, s)
          : launch_iter<__nv_bfloat16, float, true, false>(P, k, s);
    }
  }
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

// `check_every` iterations (even) followed by rr -> sc[4].
static bsp_status cg_chunk(bsp_cg_plan_s *P, cudaStream_t s) {
  for (int k = 0; k < P->opt.check_every; ++k) BSP_TRY(cg_iteration(P, k, s));
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_rr, P->grid, P->sc + 4);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

static bsp_status cg_run_chunk(bsp_cg_plan_s *P, cudaStream_t s) {
  if (!P->opt.use_graphs) return cg_chunk(P, s);
  if (!P->graph) {
    if (!P->graph_stream) BSP_CUDA(cudaStreamCreateWithFlags(&P->graph_stream, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    BSP_CUDA(cudaStreamBeginCapture(P->graph_stream, cudaStreamCaptureModeThreadLocal));
    bsp_status st = cg_chunk(P, P->graph_stream);
    cudaError_t e = cudaStreamEndCapture(P->graph_stream, &graph);
    if (st != BSP_OK) return st;
    if (e != cudaSuccess) BSP_FAIL(BSP_ERR_CUDA, cudaGetErrorString(e));
    e = cudaGraphInstantiate(&P->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) BSP_FAIL(BSP_ERR_CUDA, cudaGetErrorString(e));
  }
  BSP_CUDA(cudaGraphLaunch(P->graph, s));
  return BSP_OK;
}

static bsp_status read_scalars(bsp_cg_plan_s *P, cudaStream_t s) {
  BSP_CUDA(cudaMemcpyAsync(P->h_sc, P->sc, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

// True FP64 residual of x64 -> sc[2]; the iterated residual (and its r.r
// partials for the next iteration) is replaced by it.
// measure_dev (mixed modes): also ||r_true - r_iterated||^2 -> sc[7].
static bsp_status cg_true_residual(bsp_cg_plan_s *P, const double *b, cudaStream_t s, bool measure_dev = false) {
  const int g = P->grid;
  if (cg_mixed(P))
    cg_residual_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->x64, P->r64,
                                                        (float *)P->r, P->part_res, P->part_rr,
                                                        measure_dev ? P->part_zq : nullptr);
  else
    cg_residual_kernel<double><<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->x64,
                                                         (double *)P->r, nullptr, P->part_res, nullptr);
  BSP_LAUNCH_CHECK();
  if (!cg_mixed(P)) {  // the FP64 residual is the iterated one
    BSP_CUDA(cudaMemcpyAsync(P->part_rr, P->part_res, sizeof(double) * g, cudaMemcpyDeviceToDevice, s));
  }
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_res, g, P->sc + 2);
  BSP_LAUNCH_CHECK();
  if (measure_dev && cg_mixed(P)) {
    sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_zq, g, P->sc + 7);
    BSP_LAUNCH_CHECK();
  }
  if (P->prec_bs) {
    if (cg_mixed(P))
      launch_prec<float>(P, s);
    else
      launch_prec<double>(P, s);
    BSP_LAUNCH_CHECK();
  }
  return BSP_OK;
}

// M^{-1} (Jacobi or block-Jacobi) of the CSR matrix in the iteration precision.
template <typename VT>
static bsp_status build_minv(bsp_cg_plan_s *P, cudaStream_t s) {
  const int bs = P->prec_bs;
  const int64_t nb = ((int64_t)P->n + bs - 1) / bs;
  BSP_CUDA(cudaMallocAsync(&P->minv, sizeof(VT) * (size_t)(nb * bs * bs), s));
  int32_t *bad = nullptr;
  BSP_TRY(dalloc(&bad, 1, s));
  BSP_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  const unsigned gr = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(nb, 128), (int64_t)sm_count() * 16));
  VT *mi = (VT *)P->minv;
  if (bs == 1)
    cg_minv_kernel<VT, 1><<<gr, 128, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, mi, bad);
  else if (bs == 4)
    cg_minv_kernel<VT, 4><<<gr, 128, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, mi, bad);
  else
    cg_minv_kernel<VT, 8><<<gr, 128, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, mi, bad);
  BSP_LAUNCH_CHECK();
  int32_t h_bad = 0;
  const bsp_status st = read_i32(bad, &h_bad, s);
  dfree(bad, s);
  BSP_TRY(st);
  if (h_bad)
    BSP_FAIL(BSP_ERR_INVALID, bs == 1 ? "a diagonal entry is zero or not finite"
                                      : "a diagonal block is singular or not finite");
  return BSP_OK;
}

// Enters the flexible outer iteration from a folded state (x_lp = 0, r64 and
// r_lp = b - A x64): no previous direction, inner direction restarted.
static bsp_status fcg_begin(bsp_cg_plan_s *P, cudaStream_t s) {
  BSP_CUDA(cudaMemsetAsync(P->p64, 0, sizeof(double) * P->n, s));
  BSP_CUDA(cudaMemsetAsync(P->q64, 0, sizeof(double) * P->n, s));
  BSP_CUDA(cudaMemsetAsync(P->sc, 0, 2 * sizeof(double), s));
  BSP_CUDA(cudaMemsetAsync(P->sc + 5, 0, sizeof(double), s));
  return BSP_OK;
}

// One outer step with z = the inner solution since the last step; then the
// inner iteration restarts on the new residual.  ||r64||^2 -> sc[6].
static bsp_status fcg_step(bsp_cg_plan_s *P, cudaStream_t s) {
  const int g = P->grid;
  fcg_z_kernel<<<g, kCgThreads, 0, s>>>(P->n, (float *)P->x, P->z64, P->q64, P->part_zq);
  fcg_dir_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->part_zq, g, P->sc + 5, P->z64, P->p64);
  fcg_spmv_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, P->p64, P->q64, P->r64,
                                           P->part_pq, P->part_pr);
  fcg_update_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->part_pq, P->part_pr, g, P->sc + 5, P->x64, P->r64, P->p64,
                                             P->q64, (float *)P->r, P->part_res, P->part_rr);
  BSP_LAUNCH_CHECK();
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_res, g, P->sc + 6);
  BSP_LAUNCH_CHECK();
  BSP_CUDA(cudaMemsetAsync(P->sc, 0, 2 * sizeof(double), s));  // inner restart: beta = 0
  if (P->prec_bs) {
    launch_prec<float>(P, s);
    BSP_LAUNCH_CHECK();
  }
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_cg_default_options(bsp_cg_options *o) {
  clear_error();
  BSP_CHECK_ARG(o, "null options");
  o->mode = BSP_CG_MIXED_F16;
  o->tol = 1e-10;
  o->max_iters = 20000;
  o->check_every = 16;
  o->reliable_delta = 0.1;
  o->use_graphs = 1;
  o->precond = BSP_CG_PRECOND_NONE;
  o->precond_block = 4;
  o->refine = BSP_CG_REFINE_AUTO;
  return BSP_OK;
}

extern "C" bsp_status bsp_cg_destroy(bsp_cg_plan P) {
  clear_error();
  if (!P) return BSP_OK;
  cudaStream_t s = 0;
  if (P->graph) cudaGraphExecDestroy(P->graph);
  if (P->graph_stream) cudaStreamDestroy(P->graph_stream);
  if (P->x == P->x64) P->x = nullptr;  // FP64 mode iterates on x64 itself
  dfree(P->x64, s);
  dfree(P->r64, s);
  for (void *v : {P->x, P->r, P->p[0], P->p[1], P->q, P->lp_val, P->z, P->minv})
    if (v) cudaFreeAsync(v, s);
  dfree(P->part_rz, s);
  dfree(P->p64, s);
  dfree(P->q64, s);
  dfree(P->z64, s);
  dfree(P->part_zq, s);
  dfree(P->part_pr, s);
  if (P->lp_cols) cudaFreeAsync(P->lp_cols, s);
  dfree(P->exps, s);
  dfree(P->slice_len, s);
  dfree(P->slice_off, s);
  dfree(P->part_pq, s);
  dfree(P->part_rr, s);
  dfree(P->part_res, s);
  dfree(P->sc, s);
  if (P->h_sc) cudaFreeHost(P->h_sc);
  cudaStreamSynchronize(s);
  delete P;
  return BSP_OK;
}

extern "C" bsp_status bsp_cg_create(int32_t n, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                    const double *values, const bsp_cg_options *opt, bsp_cg_plan *out,
                                    bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out && opt, "null argument");
  BSP_CHECK_ARG(n > 0 && nnz >= 0 && rowPtr && colIdx && values, "bad matrix");
  BSP_CHECK_ARG(opt->mode >= BSP_CG_FP64 && opt->mode <= BSP_CG_MIXED_BF16, "unknown mode");
  BSP_CHECK_ARG(opt->tol > 0 && opt->check_every >= 1 && opt->max_iters >= 1, "bad options");
  BSP_CHECK_ARG(opt->reliable_delta > 0 && opt->reliable_delta < 1, "reliable_delta must be in (0, 1)");
  BSP_CHECK_ARG(opt->precond >= BSP_CG_PRECOND_NONE && opt->precond <= BSP_CG_PRECOND_BLOCK_JACOBI,
                "unknown preconditioner");
  BSP_CHECK_ARG(opt->precond != BSP_CG_PRECOND_BLOCK_JACOBI || opt->precond_block == 4 || opt->precond_block == 8,
                "precond_block must be 4 or 8");
  BSP_CHECK_ARG(opt->refine >= BSP_CG_REFINE_AUTO && opt->refine <= BSP_CG_REFINE_FLEXIBLE, "unknown refine");
  cudaStream_t s = as_stream(stream);
  bsp_cg_plan_s *P = new bsp_cg_plan_s();
  P->n = n;
  P->nnz = nnz;
  P->opt = *opt;
  P->opt.check_every += P->opt.check_every & 1;  // even: iteration parity restarts at every chunk
  P->rowPtr = rowPtr;
  P->colIdx = colIdx;
  P->val = values;
  P->grid = (int)std::min<int64_t>(ceil_div(n, kCgThreads), (int64_t)sm_count() * kCgMaxCtasPerSm);
  const bool mixed = cg_mixed(P);
  const size_t vt = mixed ? 4 : 8;
  bsp_status st = BSP_OK;
  auto fail = [&](bsp_status e) {
    bsp_cg_destroy(P);
    return e;
  };
#define BSP_CG_TRY(x)                         \
  do {                                        \
    if ((st = (x)) != BSP_OK) return fail(st); \
  } while (0)
#define BSP_CG_CUDA(x)                                                              \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) {                                                        \
      set_error(std::string("bsp_cg_create: ") + #x + " -> " + cudaGetErrorString(e_)); \
      return fail(BSP_ERR_ALLOC);                                                   \
    }                                                                               \
  } while (0)
  BSP_CG_TRY(dalloc(&P->x64, (size_t)n, s));
  BSP_CG_TRY(dalloc(&P->part_pq, (size_t)P->grid, s));
  BSP_CG_TRY(dalloc(&P->part_rr, (size_t)P->grid, s));
  BSP_CG_TRY(dalloc(&P->part_res, (size_t)P->grid, s));
  BSP_CG_TRY(dalloc(&P->sc, 8, s));
  BSP_CG_CUDA(cudaMallocHost(reinterpret_cast<void **>(&P->h_sc), 8 * sizeof(double)));
  if (mixed) {
    P->x = nullptr;  // x32 allocated below
  }
  for (void **v : {&P->x, &P->r, &P->p[0], &P->p[1], &P->q}) BSP_CG_CUDA(cudaMallocAsync(v, vt * (size_t)n, s));
  if (!mixed) {  // lanes per row from the mean row length
    const double mean = (double)nnz / n;
    P->lpr = mean <= 10.0 ? 1 : mean <= 20.0 ? 2 : mean <= 40.0 ? 4 : 8;
  }
  P->prec_bs = opt->precond == BSP_CG_PRECOND_JACOBI ? 1
               : opt->precond == BSP_CG_PRECOND_BLOCK_JACOBI ? opt->precond_block : 0;
  if (mixed) {
    BSP_CG_TRY(dalloc(&P->r64, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->p64, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->q64, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->z64, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->part_zq, (size_t)P->grid, s));
    BSP_CG_TRY(dalloc(&P->part_pr, (size_t)P->grid, s));
  }
  if (P->prec_bs) {
    BSP_CG_CUDA(cudaMallocAsync(&P->z, vt * (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->part_rz, (size_t)P->grid, s));
    BSP_CG_TRY(mixed ? build_minv<float>(P, s) : build_minv<double>(P, s));
  }
  if (!mixed) {  // FP64 mode iterates directly on x64
    cudaFreeAsync(P->x, s);
    P->x = P->x64;
  }
  int64_t mat_bytes = (int64_t)nnz * 12;
  // FP64 mode with short rows: an FP64 SELL-32 copy with 16-bit column
  // offsets (10 bytes per entry, coalesced, no row pointers) replaces the CSR
  // walk when its slices are uniform; otherwise the CSR kernel runs.
  const bool try64 = !mixed && P->lpr == 1;
  int64_t padded = 0;
  if (mixed || try64) {
    const bool scaled = mixed && opt->mode != BSP_CG_MIXED_F32;
    // SELL-32 slices: lengths on the device, offsets summed on the host
    const int64_t ns = ceil_div(n, 32);
    BSP_CG_TRY(dalloc(&P->slice_len, (size_t)ns, s));
    BSP_CG_TRY(dalloc(&P->slice_off, (size_t)ns + 1, s));
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(ns, 256), (int64_t)sm_count() * 16));
    sell_len_kernel<<<gs, 256, 0, s>>>(n, rowPtr, P->slice_len);
    std::vector<int32_t> hlen((size_t)ns);
    std::vector<int64_t> hoff((size_t)ns + 1, 0);
    BSP_CG_CUDA(cudaMemcpyAsync(hlen.data(), P->slice_len, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, s));
    BSP_CG_CUDA(cudaStreamSynchronize(s));
    // When padding every slice to the longest costs at most 1/32 more
    // storage (stencils, banded matrices), the direction kernel computes a
    // slice's offset instead of loading its length and offset.
    int32_t lmax = 0;
    int64_t natural = 0;
    for (int64_t k = 0; k < ns; ++k) {
      lmax = std::max(lmax, hlen[k]);
      natural += 32 * (int64_t)hlen[k];
    }
    if (lmax > 0 && ns * 32 * (int64_t)lmax <= natural + natural / 32) {
      std::fill(hlen.begin(), hlen.end(), lmax);
      BSP_CG_CUDA(cudaMemcpyAsync(P->slice_len, hlen.data(), sizeof(int32_t) * ns, cudaMemcpyHostToDevice, s));
      P->sell_uniform = lmax;
    }
    for (int64_t k = 0; k < ns; ++k) hoff[k + 1] = hoff[k] + 32 * (int64_t)hlen[k];
    padded = hoff[ns];
    if (padded >= ((int64_t)1 << 31)) {
      if (mixed) {
        set_error("bsp_cg_create: the padded low-precision matrix needs >= 2^31 entries");
        return fail(BSP_ERR_UNSUPPORTED);
      }
      P->sell_uniform = 0;  // FP64 stays on the CSR arrays
    }
    BSP_CG_CUDA(cudaMemcpyAsync(P->slice_off, hoff.data(), sizeof(int64_t) * (ns + 1), cudaMemcpyHostToDevice, s));
    if (scaled) {
      BSP_CG_TRY(dalloc(&P->exps, (size_t)n, s));
      const unsigned ge = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 16));
      row_exp_kernel<<<ge, 256, 0, s>>>(n, rowPtr, values, P->exps);
    }
    int32_t *bad = nullptr;
    BSP_CG_TRY(dalloc(&bad, 1, s));
    cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
    int64_t gr = ceil_div(n, 256);
    if (gr > (int64_t)sm_count() * 32) gr = (int64_t)sm_count() * 32;
    cg_delta_check_kernel<<<(unsigned)gr, 256, 0, s>>>(n, rowPtr, colIdx, bad);
    int32_t h_bad = 1;
    BSP_CG_TRY(read_i32(bad, &h_bad, s));
    dfree(bad, s);
    P->delta16 = !h_bad;
    P->sell64 = try64 && P->delta16 && P->sell_uniform > 0;
    if (try64 && !P->sell64) {  // FP64 stays on the CSR arrays
      dfree(P->slice_len, s);
      dfree(P->slice_off, s);
      P->slice_len = nullptr;
      P->slice_off = nullptr;
      P->sell_uniform = 0;
    }
  }
  if (mixed || P->sell64) {
    const bool scaled = mixed && opt->mode != BSP_CG_MIXED_F32;
    const size_t vsz = !mixed ? 8 : opt->mode == BSP_CG_MIXED_F32 ? 4 : 2;
    const bool packed = scaled && P->delta16;
    if (P->sell64) {
      // the FP64 copy is an optimisation: without room for it, stay on CSR
      const size_t ne = (size_t)(padded > 0 ? padded : 1);
      if (cudaMallocAsync(&P->lp_val, 8 * ne, s) != cudaSuccess ||
          cudaMallocAsync(&P->lp_cols, 2 * ne, s) != cudaSuccess) {
        cudaGetLastError();
        if (P->lp_val) cudaFreeAsync(P->lp_val, s);
        if (P->lp_cols) cudaFreeAsync(P->lp_cols, s);
        P->lp_val = P->lp_cols = nullptr;
        dfree(P->slice_len, s);
        dfree(P->slice_off, s);
        P->slice_len = nullptr;
        P->slice_off = nullptr;
        P->sell_uniform = 0;
        P->sell64 = false;
      }
    } else {
      BSP_CG_CUDA(cudaMallocAsync(&P->lp_val, (packed ? 4 : vsz) * (size_t)(padded > 0 ? padded : 1), s));
      if (!packed)
        BSP_CG_CUDA(cudaMallocAsync(&P->lp_cols, (P->delta16 ? 2 : 4) * (size_t)(padded > 0 ? padded : 1), s));
    }
  }
  if (mixed || P->sell64) {
    const bool scaled = mixed && opt->mode != BSP_CG_MIXED_F32;
    const size_t vsz = !mixed ? 8 : opt->mode == BSP_CG_MIXED_F32 ? 4 : 2;
    const int64_t ns = ceil_div(n, 32);
    const bool packed = scaled && P->delta16;
    int64_t gf = ceil_div(ns * 32, 256);
    if (gf > (int64_t)sm_count() * 32) gf = (int64_t)sm_count() * 32;
#define BSP_SELL_FILL(V, SC, D, PK)                                                                          \
  sell_fill_kernel<V, SC, D, PK><<<(unsigned)gf, 256, 0, s>>>(n, rowPtr, colIdx, values, P->slice_len,           \
                                                              P->slice_off, P->exps, (V *)P->lp_val, P->lp_cols)
    if (!mixed) {
      BSP_SELL_FILL(double, false, true, false);
    } else if (opt->mode == BSP_CG_MIXED_F32) {
      if (P->delta16) BSP_SELL_FILL(float, false, true, false); else BSP_SELL_FILL(float, false, false, false);
    } else if (opt->mode == BSP_CG_MIXED_F16) {
      if (P->delta16) BSP_SELL_FILL(__half, true, true, true); else BSP_SELL_FILL(__half, true, false, false);
    } else {
      if (P->delta16)
        BSP_SELL_FILL(__nv_bfloat16, true, true, true);
      else
        BSP_SELL_FILL(__nv_bfloat16, true, false, false);
    }
#undef BSP_SELL_FILL
    if (cudaGetLastError() != cudaSuccess) {
      set_error("bsp_cg_create: building the low-precision matrix failed");
      return fail(BSP_ERR_CUDA);
    }
    mat_bytes = padded * (packed ? 4 : (int64_t)vsz + (P->delta16 ? 2 : 4)) + (scaled ? (int64_t)n : 0) + 12 * ns;
  }
  {  // partials were sized for the largest grid
    int oa = 4, ob = 4;
    cg_plan_occupancy(P, oa, ob);
    P->grid_a = cg_grid(n, oa);
    P->grid = cg_grid(n, ob);
  }
#undef BSP_CG_TRY
#undef BSP_CG_CUDA
  // algorithmic bytes: kernel A reads the matrix, r and p_prev (own rows;
  // gathers counted once) and writes p and q; kernel B reads p, q, x, r and
  // writes x, r.
  // Preconditioned: the update kernel also reads M^{-1} and writes z.
  P->bytes_iter = mat_bytes + (mixed || P->sell64 ? 0 : 4 * ((int64_t)n + 1)) + 10 * (int64_t)vt * n;
  if (P->prec_bs)
    P->bytes_iter += (int64_t)vt * (ceil_div(n, P->prec_bs) * P->prec_bs * P->prec_bs + (int64_t)n);
  P->bytes_residual = (int64_t)nnz * 12 + 4 * ((int64_t)n + 1) + 3 * 8 * (int64_t)n;
  // flexible outer step: F1 8n+8n+8n, F2 24n, F3 matrix + 4(n+1) + 32n, F4 52n
  P->bytes_outer = (int64_t)nnz * 12 + 4 * ((int64_t)n + 1) + 132 * (int64_t)n;
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("bsp_cg_create: preparing the matrix failed");
    return fail(BSP_ERR_CUDA);
  }
  *out = P;
  return BSP_OK;
}

namespace bsp {
void cg_plan_view(const bsp_cg_plan_s *P, CgPlanView *v) {
  v->n = P->n;
  v->nnz = P->nnz;
  v->rowPtr = P->rowPtr;
  v->colIdx = P->colIdx;
  v->val = P->val;
  v->mixed = cg_mixed(P);
  v->prec_bs = P->prec_bs;
  v->minv = P->minv;
  v->check_every = P->opt.check_every;
  v->max_iters = P->opt.max_iters;
  v->tol = P->opt.tol;
}
}  // namespace bsp

extern "C" bsp_status bsp_cg_solve(bsp_cg_plan P, const double *b, double *x, bsp_cg_result *res,
                                   bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P && b && x && res, "null argument");
  cudaStream_t s = as_stream(stream);
  *res = bsp_cg_result{};
  const int g = P->grid;
  const bool mixed = cg_mixed(P);
  const size_t vt = mixed ? 4 : 8;
  cudaEvent_t e0, e1;
  BSP_CUDA(cudaEventCreate(&e0));
  BSP_CUDA(cudaEventCreate(&e1));
  BSP_CUDA(cudaEventRecord(e0, s));
  // ||b||^2 via the residual of x = 0 (x64 zeroed), then x64 = x0
  BSP_CUDA(cudaMemsetAsync(P->x64, 0, sizeof(double) * P->n, s));
  cg_residual_kernel<double><<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->x64, nullptr,
                                                       nullptr, P->part_res, nullptr);
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_res, g, P->sc + 3);
  BSP_LAUNCH_CHECK();
  BSP_CUDA(cudaMemcpyAsync(P->x64, x, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, s));
  // start: iterated residual, p_prev = 0, rr_prev = 0 (beta_0 = 0)
  if (mixed) BSP_CUDA(cudaMemsetAsync(P->x, 0, vt * P->n, s));
  BSP_CUDA(cudaMemsetAsync(P->p[0], 0, vt * P->n, s));
  BSP_CUDA(cudaMemsetAsync(P->sc, 0, 2 * sizeof(double), s));
  BSP_TRY(cg_true_residual(P, b, s));
  BSP_TRY(read_scalars(P, s));
  const double bb = P->h_sc[3];
  const double target = P->opt.tol * P->opt.tol * bb;
  const double delta2 = P->opt.reliable_delta * P->opt.reliable_delta;
  double rmax2 = P->h_sc[2];
  int64_t residuals = 2, iters = 0;
  int32_t updates = 0, no_progress = 0;
  double best_true = P->h_sc[2];
  bool coarse = false;
  bool done = bb == 0.0 || P->h_sc[2] <= target;
  bool flex = mixed && P->opt.refine == BSP_CG_REFINE_FLEXIBLE;
  int32_t outer = 0;
  if (flex) BSP_TRY(fcg_begin(P, s));
  // replacements / outer steps that stop lowering the residual: the
  // low-precision copy is too coarse for this matrix
  auto progress = [&](double r2) {
    if (r2 < best_true) {
      best_true = r2;
      no_progress = 0;
    } else if (++no_progress >= kCgNoProgress) {
      coarse = true;
    }
  };
  int chunks = 0;  // since the last replacement / outer step
  while (!done && iters < P->opt.max_iters) {
    BSP_TRY(cg_run_chunk(P, s));
    iters += P->opt.check_every;
    ++chunks;
    BSP_TRY(read_scalars(P, s));
    const double rr = P->h_sc[4];
    const bool stalled = !(rr == rr);  // NaN
    const bool growing = mixed && (rr > kCgGrowth * rmax2 || chunks >= kCgInnerChunks);
    if (!(rr <= target || (mixed && rr <= delta2 * rmax2) || stalled || growing)) continue;
    chunks = 0;
    if (flex) {
      if (stalled) break;
      BSP_TRY(fcg_step(P, s));
      BSP_TRY(read_scalars(P, s));
      ++outer;
      double r2 = P->h_sc[6];
      if (r2 <= target) {  // confirm with the true residual (which also restarts the inner iteration)
        BSP_TRY(cg_true_residual(P, b, s));
        BSP_CUDA(cudaMemsetAsync(P->sc, 0, 2 * sizeof(double), s));
        BSP_TRY(read_scalars(P, s));
        ++residuals;
        r2 = P->h_sc[2];
      }
      rmax2 = r2;
      progress(r2);
      done = r2 <= target || coarse;
      continue;
    }
    // reliable update: fold the inner solution, replace the residual
    if (mixed) {
      cg_fold_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, (float *)P->x, P->x64);
      BSP_LAUNCH_CHECK();
    }
    BSP_TRY(cg_true_residual(P, b, s, mixed));
    BSP_TRY(read_scalars(P, s));
    ++residuals;
    ++updates;
    // A true residual far (in direction, not only in norm) from the iterated
    // one it replaces: the low-precision matrix is far from A (a large
    // condition number times the storage rounding) and the kept direction no
    // longer fits the replaced residual.  AUTO switches to the flexible outer
    // iteration; RELIABLE restarts the direction (beta = 0, i.e. iterative
    // refinement with CG as the inner solver).
    if (mixed && (growing || P->h_sc[7] > kCgDeviation * kCgDeviation * rr)) {
      if (P->opt.refine == BSP_CG_REFINE_AUTO) {
        flex = true;
        BSP_TRY(fcg_begin(P, s));
      } else {
        BSP_CUDA(cudaMemsetAsync(P->sc, 0, 2 * sizeof(double), s));
      }
    }
    rmax2 = P->h_sc[2];
    progress(P->h_sc[2]);
    done = P->h_sc[2] <= target || stalled || coarse;
  }
  if (!done && mixed) {  // budget spent: apply what the inner solve has
    if (flex) {
      BSP_TRY(fcg_step(P, s));
      ++outer;
    } else {
      cg_fold_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, (float *)P->x, P->x64);
      BSP_LAUNCH_CHECK();
    }
    BSP_TRY(cg_true_residual(P, b, s));
    ++residuals;
  }
  BSP_CUDA(cudaMemcpyAsync(x, P->x64, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, s));
  BSP_CUDA(cudaEventRecord(e1, s));
  BSP_TRY(read_scalars(P, s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  res->iterations = (int32_t)iters;
  res->reliable_updates = updates;
  res->outer_steps = outer;
  res->seconds = ms * 1e-3;
  res->rel_residual = bb > 0 ? sqrt(P->h_sc[2] / bb) : 0.0;
  res->converged = res->rel_residual <= P->opt.tol;
  res->bytes_moved = residuals * P->bytes_residual + iters * P->bytes_iter + (int64_t)outer * P->bytes_outer;
  res->delta16 = P->delta16 ? 1 : 0;
  if (!res->converged) {
    set_error("CG stopped at relative residual " + std::to_string(res->rel_residual) +
              (coarse ? ": the low-precision matrix is too coarse for this matrix's condition number "
                        "(residual replacements stopped reducing the residual); use mode f32 or fp64"
                      : ""));
    return BSP_ERR_NOT_CONVERGED;
  }
  return BSP_OK;
}
