// Conjugate gradients on the device: plain FP64 CG and mixed-precision CG
// with FP64 iterative refinement.  The reference has no solver (SURVEY: the
// CG / mixed-precision rows are absent there); this is the precision form of
// the benchmark's CG configuration: 3-D 7-point Poisson, tolerance 1e-10 on
// ||b - A x|| / ||b|| checked in FP64.
//
// Mixed precision: the matrix is stored a second time with values in FP32,
// FP16 or BF16.  FP16/BF16 values carry one power-of-two exponent per group of
// 32 consecutive nonzeros (v = stored * 2^e, the group maximum scaled into
// [1, 2)), and column indices are stored as int16 offsets from the row when
// every |col - row| < 32768 (banded matrices), else int32.  A nonzero then
// moves 4 bytes (FP16/BF16 + int16) instead of 12 (FP64 + int32).  The outer
// loop keeps r = b - A x, ||r|| and x += d in FP64 with the FP64 matrix; the
// inner CG solves A d = r / ||r|| in FP32 vectors to a relative tolerance,
// with FP64 dot products.
//
// Kernels per CG iteration (one CUDA graph captures `check_every`
// iterations; the host reads the residual between graphs):
//   1. q = A p fused with per-CTA partials of p.q;
//   2. alpha = rr / p.q (every CTA reduces the partials in the same order:
//      deterministic, no atomics), x += alpha p, r -= alpha q, partials of r.r;
//   3. beta = rr_new / rr, p = r + beta p (CTA 0 records rr_new).
// Zero denominators freeze the iteration (alpha = beta = 0), so iterations
// run after convergence inside a graph are harmless.
#include <math.h>

#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

constexpr int kCgThreads = 256;
constexpr int kScaleGroup = 32;

template <typename V> __device__ __forceinline__ float lp_to_float(V v);
template <> __device__ __forceinline__ float lp_to_float<float>(float v) { return v; }
template <> __device__ __forceinline__ float lp_to_float<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float lp_to_float<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// 2^e as a float built from its exponent bits (|e| <= 126).
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }

// Deterministic block sum of one double per thread (fixed shuffle tree, then
// warp totals in order).  Result valid in thread 0.
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

// Sum of the n partials in index order; every CTA gets the same value.
__device__ __forceinline__ double reduce_partials(const double *__restrict__ part, int n, double *smem) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kCgThreads) s += __ldcg(part + i);
  s = block_sum(s, smem);
  __shared__ double bcast;
  if (threadIdx.x == 0) bcast = s;
  __syncthreads();
  return bcast;
}

// q = A p and partial p.q.  Matrix values V (double, float, half, bf16),
// optional group exponents, int32 columns or int16 offsets from the row.
// Vectors VT (double for FP64 CG, float for the inner solve).  LPR lanes per row.
template <typename V, typename VT, bool SCALED, bool DELTA16, int LPR>
__global__ void __launch_bounds__(kCgThreads) cg_spmv_dot_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                                 const void *__restrict__ cols,
                                                                 const V *__restrict__ val,
                                                                 const int8_t *__restrict__ exps,
                                                                 const VT *__restrict__ p, VT *__restrict__ q,
                                                                 double *__restrict__ part) {
  __shared__ double smem[kCgThreads / 32];
  const int sub = threadIdx.x & (LPR - 1);
  const int64_t groups = (int64_t)gridDim.x * (kCgThreads / LPR);
  double dot = 0.0;
  const int64_t warp_first = ((int64_t)blockIdx.x * kCgThreads + (threadIdx.x & ~31)) / LPR;
  for (int64_t base = warp_first; base < n; base += groups) {
    const int64_t r = base + (threadIdx.x & 31) / LPR;
    const bool active = r < n;
    const int32_t s = active ? rowPtr[r] : 0, e = active ? rowPtr[r + 1] : 0;
    VT acc = VT(0);
    for (int32_t j = s + sub; j < e; j += LPR) {
      int64_t c;
      if (DELTA16)
        c = r + (int64_t) reinterpret_cast<const int16_t *>(cols)[j];
      else
        c = reinterpret_cast<const int32_t *>(cols)[j];
      VT a;
      if constexpr (sizeof(V) == 8) {
        a = (VT)val[j];
      } else {
        float af = lp_to_float<V>(val[j]);
        if (SCALED) af *= pow2f(exps[j / kScaleGroup]);
        a = (VT)af;
      }
      acc = fma(a, __ldg(p + c), acc);
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, LPR);
    if (active && sub == 0) {
      q[r] = acc;
      dot += (double)acc * (double)p[r];
    }
  }
  const double t = block_sum(dot, smem);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// r = b - A x and partial ||r||^2, all FP64 (outer refinement / FP64 CG start).
__global__ void __launch_bounds__(kCgThreads) cg_residual_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                                 const int32_t *__restrict__ colIdx,
                                                                 const double *__restrict__ val,
                                                                 const double *__restrict__ b,
                                                                 const double *__restrict__ x,
                                                                 double *__restrict__ r, double *__restrict__ part) {
  __shared__ double smem[kCgThreads / 32];
  constexpr int LPR = 8;
  const int sub = threadIdx.x & (LPR - 1);
  const int64_t groups = (int64_t)gridDim.x * (kCgThreads / LPR);
  double nrm = 0.0;
  const int64_t warp_first = ((int64_t)blockIdx.x * kCgThreads + (threadIdx.x & ~31)) / LPR;
  for (int64_t base = warp_first; base < n; base += groups) {
    const int64_t i = base + (threadIdx.x & 31) / LPR;
    const bool active = i < n;
    const int32_t s = active ? rowPtr[i] : 0, e = active ? rowPtr[i + 1] : 0;
    double acc = 0.0;
    for (int32_t j = s + sub; j < e; j += LPR) acc = fma(val[j], __ldg(x + colIdx[j]), acc);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, LPR);
    if (active && sub == 0) {
      const double ri = b[i] - acc;
      r[i] = ri;
      nrm += ri * ri;
    }
  }
  const double t = block_sum(nrm, smem);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Scalars kept on the device (sc[]): [0], [1] = r.r of even / odd iterations
// (ping-pong: iteration k reads slot k%2 and writes slot (k+1)%2, so no CTA
// can see a value written in its own launch), [2] = r.r at the start,
// [3] = iterations, [4] = ||b||^2, [5] = ||b - A x||^2 of the last residual.
// alpha = rr / pq; x += alpha p; r -= alpha q; partial r.r.
template <typename VT>
__global__ void __launch_bounds__(kCgThreads) cg_update_kernel(int32_t n, const double *__restrict__ pq_part,
                                                               int npart, const double *__restrict__ rr_slot,
                                                               VT *__restrict__ x, VT *__restrict__ r,
                                                               const VT *__restrict__ p, const VT *__restrict__ q,
                                                               double *__restrict__ rr_part) {
  __shared__ double smem[kCgThreads / 32];
  const double pq = reduce_partials(pq_part, npart, smem);
  const double rr = *rr_slot;
  const double alpha = (pq != 0.0 && rr != 0.0 && isfinite(pq)) ? rr / pq : 0.0;
  const VT a = (VT)alpha;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    x[i] = fma(a, p[i], x[i]);
    const VT ri = fma(-a, q[i], r[i]);
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  const double t = block_sum(s, smem);
  if (threadIdx.x == 0) rr_part[blockIdx.x] = t;
}

// beta = rr_new / rr; p = r + beta p; CTA 0 stores rr_new in the other slot.
template <typename VT>
__global__ void __launch_bounds__(kCgThreads) cg_direction_kernel(int32_t n, const double *__restrict__ rr_part,
                                                                  int npart, const double *__restrict__ rr_slot,
                                                                  double *__restrict__ rr_next,
                                                                  double *__restrict__ sc,
                                                                  const VT *__restrict__ r, VT *__restrict__ p) {
  __shared__ double smem[kCgThreads / 32];
  const double rr_new = reduce_partials(rr_part, npart, smem);
  const double rr = *rr_slot;
  const double beta = (rr != 0.0 && isfinite(rr_new)) ? rr_new / rr : 0.0;
  const VT bt = (VT)beta;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads)
    p[i] = fma(bt, p[i], r[i]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *rr_next = rr_new;
    sc[3] += 1.0;
  }
}

// Start of a (inner or FP64) CG: r given, p = r, rr = r.r from partials, x = 0.
template <typename VT>
__global__ void __launch_bounds__(kCgThreads) cg_start_kernel(int32_t n, const double *__restrict__ rr_part,
                                                              int npart, double *__restrict__ sc,
                                                              const VT *__restrict__ r, VT *__restrict__ p,
                                                              VT *__restrict__ x, int zero_x) {
  __shared__ double smem[kCgThreads / 32];
  const double rr = reduce_partials(rr_part, npart, smem);
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    p[i] = r[i];
    if (zero_x) x[i] = VT(0);
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc[0] = rr;
    sc[2] = rr;
    sc[3] = 0.0;
  }
}

// Inner start from the FP64 residual: r32 = r64 / ||r64||, partial r32.r32.
__global__ void __launch_bounds__(kCgThreads) cg_scale_rhs_kernel(int32_t n, const double *__restrict__ r64,
                                                                  const double *__restrict__ nrm2_p,
                                                                  float *__restrict__ r32,
                                                                  double *__restrict__ rr_part) {
  __shared__ double smem[kCgThreads / 32];
  const double nrm2 = *nrm2_p;
  const double inv = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads) {
    const float v = (float)(r64[i] * inv);
    r32[i] = v;
    s += (double)v * (double)v;
  }
  const double t = block_sum(s, smem);
  if (threadIdx.x == 0) rr_part[blockIdx.x] = t;
}

// x64 += ||r64|| * d32 (refinement update).
__global__ void cg_refine_kernel(int32_t n, const double *__restrict__ nrm2_p, const float *__restrict__ d,
                                 double *__restrict__ x) {
  const double nrm = sqrt(*nrm2_p);
  for (int64_t i = (int64_t)blockIdx.x * kCgThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kCgThreads)
    x[i] = fma(nrm, (double)d[i], x[i]);
}

__global__ void sum_partials_kernel(const double *__restrict__ part, int npart, double *__restrict__ out) {
  __shared__ double smem[kCgThreads / 32];
  const double s = reduce_partials(part, npart, smem);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Low-precision copy of the matrix.
__global__ void cg_group_exp_kernel(int64_t nnz, const double *__restrict__ val, int8_t *__restrict__ exps) {
  const int64_t ng = (nnz + kScaleGroup - 1) / kScaleGroup;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
    double m = 0.0;
    for (int64_t j = g * kScaleGroup; j < nnz && j < (g + 1) * kScaleGroup; ++j) m = fmax(m, fabs(val[j]));
    int e = 0;
    if (m > 0.0) {
      frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
      e -= 1;        // scaled group maximum in [1, 2)
    }
    e = e < -100 ? -100 : (e > 100 ? 100 : e);
    exps[g] = (int8_t)e;
  }
}

template <typename V>
__device__ __forceinline__ V from_float_lp(float f);
template <> __device__ __forceinline__ float from_float_lp<float>(float f) { return f; }
template <> __device__ __forceinline__ __half from_float_lp<__half>(float f) { return __float2half_rn(f); }
template <> __device__ __forceinline__ __nv_bfloat16 from_float_lp<__nv_bfloat16>(float f) { return __float2bfloat16_rn(f); }

template <typename V, bool SCALED>
__global__ void cg_quantize_kernel(int64_t nnz, const double *__restrict__ val, const int8_t *__restrict__ exps,
                                   V *__restrict__ out) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x) {
    double v = val[j];
    if (SCALED) v = ldexp(v, -(int)exps[j / kScaleGroup]);
    out[j] = from_float_lp<V>((float)v);
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

__global__ void cg_delta_fill_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                     const int32_t *__restrict__ colIdx, int16_t *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; ++j) out[j] = (int16_t)((int64_t)colIdx[j] - i);
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
  // low-precision copy
  void *lp_val = nullptr;
  int8_t *exps = nullptr;
  void *lp_cols = nullptr;  // int16 offsets or nullptr (then colIdx)
  bool delta16 = false;
  // vectors
  double *r64 = nullptr, *p64 = nullptr, *q64 = nullptr, *x64 = nullptr;
  float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr;
  double *part_a = nullptr, *part_b = nullptr, *sc = nullptr, *h_sc = nullptr;
  int grid = 0;
  cudaGraphExec_t graph64 = nullptr, graph32 = nullptr;
  cudaStream_t graph_stream = nullptr;
  int64_t bytes_inner_iter = 0, bytes_fp64_iter = 0, bytes_residual = 0;
};

namespace bsp {

static int cg_grid(int32_t n) {
  int64_t g = ceil_div(n, kCgThreads);
  const int64_t cap = (int64_t)sm_count() * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Launches q = A p (+ partials) for the plan's matrix in precision `inner`.
static bsp_status launch_spmv_dot(bsp_cg_plan_s *P, bool inner, cudaStream_t s) {
  const int g = P->grid;
  if (!inner) {
    cg_spmv_dot_kernel<double, double, false, false, 8><<<g, kCgThreads, 0, s>>>(
        P->n, P->rowPtr, P->colIdx, P->val, nullptr, P->p64, P->q64, P->part_a);
    BSP_LAUNCH_CHECK();
    return BSP_OK;
  }
  const void *cols = P->delta16 ? P->lp_cols : (const void *)P->colIdx;
#define BSP_CG_LAUNCH(V, SC)                                                                             \
  do {                                                                                                   \
    if (P->delta16)                                                                                      \
      cg_spmv_dot_kernel<V, float, SC, true, 8><<<g, kCgThreads, 0, s>>>(                                \
          P->n, P->rowPtr, cols, (const V *)P->lp_val, P->exps, P->p32, P->q32, P->part_a);              \
    else                                                                                                 \
      cg_spmv_dot_kernel<V, float, SC, false, 8><<<g, kCgThreads, 0, s>>>(                               \
          P->n, P->rowPtr, cols, (const V *)P->lp_val, P->exps, P->p32, P->q32, P->part_a);              \
  } while (0)
  switch (P->opt.mode) {
    case BSP_CG_MIXED_F32: BSP_CG_LAUNCH(float, false); break;
    case BSP_CG_MIXED_F16: BSP_CG_LAUNCH(__half, true); break;
    case BSP_CG_MIXED_BF16: BSP_CG_LAUNCH(__nv_bfloat16, true); break;
    default: BSP_FAIL(BSP_ERR_INVALID, "unknown CG mode");
  }
#undef BSP_CG_LAUNCH
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

// One CG iteration (3 launches) on the inner (FP32) or FP64 vectors; `k`
// selects the r.r slot (iteration parity).
static bsp_status cg_iteration(bsp_cg_plan_s *P, bool inner, int k, cudaStream_t s) {
  BSP_TRY(launch_spmv_dot(P, inner, s));
  const int g = P->grid;
  const double *cur = P->sc + (k & 1);
  double *next = P->sc + ((k + 1) & 1);
  if (inner) {
    cg_update_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, P->part_a, g, cur, P->x32, P->r32, P->p32, P->q32,
                                                      P->part_b);
    cg_direction_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, P->part_b, g, cur, next, P->sc, P->r32, P->p32);
  } else {
    cg_update_kernel<double><<<g, kCgThreads, 0, s>>>(P->n, P->part_a, g, cur, P->x64, P->r64, P->p64, P->q64,
                                                       P->part_b);
    cg_direction_kernel<double><<<g, kCgThreads, 0, s>>>(P->n, P->part_b, g, cur, next, P->sc, P->r64, P->p64);
  }
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

// Builds (once per precision) a graph of `check_every` iterations (an even
// count, so r.r is back in slot 0 after every graph).
static bsp_status cg_graph(bsp_cg_plan_s *P, bool inner, cudaGraphExec_t *exec) {
  if (!P->graph_stream) BSP_CUDA(cudaStreamCreateWithFlags(&P->graph_stream, cudaStreamNonBlocking));
  cudaStream_t cs = P->graph_stream;
  cudaGraph_t graph = nullptr;
  BSP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  bsp_status st = BSP_OK;
  for (int k = 0; k < P->opt.check_every && st == BSP_OK; ++k) st = cg_iteration(P, inner, k, cs);
  cudaError_t e = cudaStreamEndCapture(cs, &graph);
  if (st != BSP_OK) return st;
  if (e != cudaSuccess) BSP_FAIL(BSP_ERR_CUDA, cudaGetErrorString(e));
  e = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) BSP_FAIL(BSP_ERR_CUDA, cudaGetErrorString(e));
  return BSP_OK;
}

static bsp_status read_scalars(bsp_cg_plan_s *P, cudaStream_t s) {
  BSP_CUDA(cudaMemcpyAsync(P->h_sc, P->sc, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

// Runs CG iterations (graph chunks) until r.r <= rel_tol^2 * r.r(start) or the
// budget is spent.  Returns the iterations executed.
static bsp_status cg_loop(bsp_cg_plan_s *P, bool inner, double rel_tol, int32_t max_iters, int32_t *iters,
                          cudaStream_t s) {
  *iters = 0;
  BSP_TRY(read_scalars(P, s));
  const double target = rel_tol * rel_tol * P->h_sc[2];
  if (P->h_sc[0] <= target) return BSP_OK;
  cudaGraphExec_t *exec = inner ? &P->graph32 : &P->graph64;
  if (P->opt.use_graphs && !*exec) BSP_TRY(cg_graph(P, inner, exec));
  while (*iters < max_iters) {
    if (P->opt.use_graphs) {
      BSP_CUDA(cudaGraphLaunch(*exec, s));
    } else {
      for (int k = 0; k < P->opt.check_every; ++k) BSP_TRY(cg_iteration(P, inner, k, s));
    }
    *iters += P->opt.check_every;
    BSP_TRY(read_scalars(P, s));
    if (!(P->h_sc[0] > target)) break;  // also stops on NaN
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
  o->inner_tol = 1e-4;
  o->max_outer = 30;
  o->use_graphs = 1;
  return BSP_OK;
}

extern "C" bsp_status bsp_cg_create(int32_t n, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                                    const double *values, const bsp_cg_options *opt, bsp_cg_plan *out,
                                    bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out && opt, "null argument");
  BSP_CHECK_ARG(n > 0 && nnz >= 0 && rowPtr && colIdx && values, "bad matrix");
  BSP_CHECK_ARG(opt->mode >= BSP_CG_FP64 && opt->mode <= BSP_CG_MIXED_BF16, "unknown mode");
  BSP_CHECK_ARG(opt->tol > 0 && opt->check_every >= 1 && opt->max_iters >= 1 && opt->max_outer >= 1,
                "bad options");
  BSP_CHECK_ARG(opt->inner_tol > 0 && opt->inner_tol < 1, "inner_tol must be in (0, 1)");
  cudaStream_t s = as_stream(stream);
  bsp_cg_plan_s *P = new bsp_cg_plan_s();
  P->n = n;
  P->nnz = nnz;
  P->opt = *opt;
  P->opt.check_every += P->opt.check_every & 1;  // even: r.r ends in slot 0
  P->rowPtr = rowPtr;
  P->colIdx = colIdx;
  P->val = values;
  P->grid = cg_grid(n);
  auto fail = [&](bsp_status st) {
    bsp_cg_destroy(P);
    return st;
  };
  bsp_status st;
#define BSP_CG_TRY(x)                 \
  do {                                \
    if ((st = (x)) != BSP_OK) return fail(st); \
  } while (0)
  BSP_CG_TRY(dalloc(&P->r64, (size_t)n, s));
  BSP_CG_TRY(dalloc(&P->p64, (size_t)n, s));
  BSP_CG_TRY(dalloc(&P->q64, (size_t)n, s));
  BSP_CG_TRY(dalloc(&P->x64, (size_t)n, s));
  BSP_CG_TRY(dalloc(&P->part_a, (size_t)P->grid, s));
  BSP_CG_TRY(dalloc(&P->part_b, (size_t)P->grid, s));
  BSP_CG_TRY(dalloc(&P->sc, 8, s));
  if (cudaMallocHost(reinterpret_cast<void **>(&P->h_sc), 8 * sizeof(double)) != cudaSuccess)
    return fail(BSP_ERR_ALLOC);
  const int64_t vb = 8;  // FP64 vector bytes
  P->bytes_residual = (int64_t)nnz * 12 + 4 * ((int64_t)n + 1) + 3 * vb * n;
  P->bytes_fp64_iter = (int64_t)nnz * 12 + 4 * ((int64_t)n + 1) + 3 * vb * n /* spmv: p gathers, q, p */ +
                       6 * vb * n /* update */ + 3 * vb * n /* direction */;
  if (opt->mode != BSP_CG_FP64) {
    BSP_CG_TRY(dalloc(&P->x32, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->r32, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->p32, (size_t)n, s));
    BSP_CG_TRY(dalloc(&P->q32, (size_t)n, s));
    const bool scaled = opt->mode != BSP_CG_MIXED_F32;
    const size_t vsz = opt->mode == BSP_CG_MIXED_F32 ? 4 : 2;
    if (cudaMallocAsync(&P->lp_val, vsz * (size_t)(nnz > 0 ? nnz : 1), s) != cudaSuccess) return fail(BSP_ERR_ALLOC);
    int64_t gq = ceil_div(nnz, 256);
    if (gq > (int64_t)sm_count() * 32) gq = (int64_t)sm_count() * 32;
    if (gq < 1) gq = 1;
    if (scaled) {
      const int64_t ng = ceil_div(nnz, kScaleGroup);
      BSP_CG_TRY(dalloc(&P->exps, (size_t)(ng > 0 ? ng : 1), s));
      cg_group_exp_kernel<<<(unsigned)ceil_div(ng > 0 ? ng : 1, 256), 256, 0, s>>>(nnz, values, P->exps);
    }
    if (opt->mode == BSP_CG_MIXED_F32)
      cg_quantize_kernel<float, false><<<(unsigned)gq, 256, 0, s>>>(nnz, values, nullptr, (float *)P->lp_val);
    else if (opt->mode == BSP_CG_MIXED_F16)
      cg_quantize_kernel<__half, true><<<(unsigned)gq, 256, 0, s>>>(nnz, values, P->exps, (__half *)P->lp_val);
    else
      cg_quantize_kernel<__nv_bfloat16, true><<<(unsigned)gq, 256, 0, s>>>(nnz, values, P->exps,
                                                                           (__nv_bfloat16 *)P->lp_val);
    if (cudaPeekAtLastError() != cudaSuccess) return fail(BSP_ERR_CUDA);
    // int16 column offsets when every |col - row| fits
    int32_t *bad = nullptr;
    BSP_CG_TRY(dalloc(&bad, 1, s));
    cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
    int64_t gr = ceil_div(n, 256);
    if (gr > (int64_t)sm_count() * 32) gr = (int64_t)sm_count() * 32;
    cg_delta_check_kernel<<<(unsigned)gr, 256, 0, s>>>(n, rowPtr, colIdx, bad);
    int32_t h_bad = 1;
    BSP_CG_TRY(read_i32(bad, &h_bad, s));
    dfree(bad, s);
    if (!h_bad) {
      int16_t *d16 = nullptr;
      BSP_CG_TRY(dalloc(&d16, (size_t)(nnz > 0 ? nnz : 1), s));
      cg_delta_fill_kernel<<<(unsigned)gr, 256, 0, s>>>(n, rowPtr, colIdx, d16);
      P->lp_cols = d16;
      P->delta16 = true;
    }
    const int64_t ib = P->delta16 ? 2 : 4;
    P->bytes_inner_iter = (int64_t)nnz * ((int64_t)vsz + ib) + (scaled ? ceil_div(nnz, kScaleGroup) : 0) +
                          4 * ((int64_t)n + 1) + 3 * 4 * (int64_t)n + 6 * 4 * (int64_t)n + 3 * 4 * (int64_t)n;
  }
#undef BSP_CG_TRY
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(BSP_ERR_CUDA);
  *out = P;
  return BSP_OK;
}

extern "C" bsp_status bsp_cg_destroy(bsp_cg_plan P) {
  clear_error();
  if (!P) return BSP_OK;
  cudaStream_t s = 0;
  if (P->graph64) cudaGraphExecDestroy(P->graph64);
  if (P->graph32) cudaGraphExecDestroy(P->graph32);
  if (P->graph_stream) cudaStreamDestroy(P->graph_stream);
  dfree(P->r64, s);
  dfree(P->p64, s);
  dfree(P->q64, s);
  dfree(P->x64, s);
  dfree(P->x32, s);
  dfree(P->r32, s);
  dfree(P->p32, s);
  dfree(P->q32, s);
  dfree(P->part_a, s);
  dfree(P->part_b, s);
  dfree(P->sc, s);
  if (P->lp_val) cudaFreeAsync(P->lp_val, s);
  if (P->lp_cols) cudaFreeAsync(P->lp_cols, s);
  dfree(P->exps, s);
  if (P->h_sc) cudaFreeHost(P->h_sc);
  cudaStreamSynchronize(s);
  delete P;
  return BSP_OK;
}

extern "C" bsp_status bsp_cg_solve(bsp_cg_plan P, const double *b, double *x, bsp_cg_result *res,
                                   bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P && b && x && res, "null argument");
  cudaStream_t s = as_stream(stream);
  *res = bsp_cg_result{};
  const int g = P->grid;
  cudaEvent_t e0, e1;
  BSP_CUDA(cudaEventCreate(&e0));
  BSP_CUDA(cudaEventCreate(&e1));
  BSP_CUDA(cudaEventRecord(e0, s));
  // x64 = initial guess; ||b||^2 from the residual of x = 0 (q64 as zero vector)
  BSP_CUDA(cudaMemcpyAsync(P->x64, x, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, s));
  BSP_CUDA(cudaMemsetAsync(P->q64, 0, sizeof(double) * P->n, s));
  cg_residual_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->q64, P->r64, P->part_a);
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_a, g, P->sc + 4);
  BSP_LAUNCH_CHECK();
  BSP_TRY(read_scalars(P, s));
  const double bb = P->h_sc[4];
  int64_t spmv_fp64 = 1, spmv_inner = 0, fp64_iters = 0;
  int32_t total = 0;
  const bool inner = P->opt.mode != BSP_CG_FP64;
  for (int outer = 0; bb > 0.0 && outer < P->opt.max_outer; ++outer) {
    // FP64 true residual r = b - A x and ||r||^2 -> sc[5]
    cg_residual_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->x64, P->r64,
                                                 P->part_a);
    sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_a, g, P->sc + 5);
    BSP_LAUNCH_CHECK();
    spmv_fp64++;
    BSP_TRY(read_scalars(P, s));
    res->outer_iterations = outer;
    if (P->h_sc[5] <= P->opt.tol * P->opt.tol * bb) break;
    if (total >= P->opt.max_iters) break;
    int32_t it = 0;
    if (inner) {
      // solve A d = r / ||r|| in the inner precision, then x += ||r|| d
      cg_scale_rhs_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->r64, P->sc + 5, P->r32, P->part_b);
      cg_start_kernel<float><<<g, kCgThreads, 0, s>>>(P->n, P->part_b, g, P->sc, P->r32, P->p32, P->x32, 1);
      BSP_LAUNCH_CHECK();
      BSP_TRY(cg_loop(P, true, P->opt.inner_tol, P->opt.max_iters - total, &it, s));
      cg_refine_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->sc + 5, P->x32, P->x64);
      BSP_LAUNCH_CHECK();
      spmv_inner += it;
    } else {
      // FP64 CG from the current x (restarted with the true residual when the
      // recursive one has converged but the true one has not)
      cg_start_kernel<double><<<g, kCgThreads, 0, s>>>(P->n, P->part_a, g, P->sc, P->r64, P->p64, P->x64, 0);
      BSP_LAUNCH_CHECK();
      const double rel = P->opt.tol * sqrt(bb / P->h_sc[5]);
      BSP_TRY(cg_loop(P, false, rel < 1.0 ? rel : 1.0, P->opt.max_iters - total, &it, s));
      fp64_iters += it;
    }
    total += it;
    res->outer_iterations = outer + 1;
  }
  BSP_CUDA(cudaMemcpyAsync(x, P->x64, sizeof(double) * P->n, cudaMemcpyDeviceToDevice, s));
  // the last residual in sc[5] is the true FP64 residual of the returned x
  // unless the loop ran out; recompute it to report it exactly
  cg_residual_kernel<<<g, kCgThreads, 0, s>>>(P->n, P->rowPtr, P->colIdx, P->val, b, P->x64, P->r64, P->part_a);
  sum_partials_kernel<<<1, kCgThreads, 0, s>>>(P->part_a, g, P->sc + 5);
  BSP_LAUNCH_CHECK();
  BSP_CUDA(cudaEventRecord(e1, s));
  BSP_TRY(read_scalars(P, s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  res->iterations = total;
  res->seconds = ms * 1e-3;
  res->rel_residual = bb > 0 ? sqrt(P->h_sc[5] / bb) : 0.0;
  res->converged = res->rel_residual <= P->opt.tol;
  res->bytes_moved = spmv_fp64 * P->bytes_residual + fp64_iters * P->bytes_fp64_iter + spmv_inner * P->bytes_inner_iter;
  res->delta16 = P->delta16 ? 1 : 0;
  if (!res->converged) {
    set_error("CG stopped at relative residual " + std::to_string(res->rel_residual));
    return BSP_ERR_NOT_CONVERGED;
  }
  return BSP_OK;
}
