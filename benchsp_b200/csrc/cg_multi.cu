// CG for several right-hand sides at once (A X = B, k <= 8 columns per
// pass; no counterpart in the reference, which has no solver).
//
// Every column runs its own CG (own alpha, beta; the iterates are those of k
// separate FP64 CGs), but one pass over the matrix serves all of them: the
// blocks X, R, Z, P, Q are row-major n x K (K = 2, 4 or 8 >= k, padded
// columns zero and frozen), so a gathered row of the direction block is K
// consecutive doubles, read by K / 2 lanes with one 16-byte access each, and
// the matrix entry is read once for K products.  An iteration is the same two kernels as the single-vector
// solver:
//   A. beta_j = rz_j / rz_prev_j; P = Z + beta (.) P_prev formed for every
//      gathered row; Q = A P; partials of p_j.q_j;
//   B. alpha_j = rz_j / p_j.q_j; X += alpha (.) P; R -= alpha (.) Q;
//      Z = D^{-1} R (Jacobi) or Z = R; partials of r_j.r_j and r_j.z_j.
// Per-CTA partials are reduced in a fixed order by every CTA (deterministic);
// a zero or non-finite denominator freezes that column.
#include <algorithm>
#include <cmath>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {
namespace {

constexpr int kMcgThreads = 256;

__device__ __forceinline__ double mcg_block_sum(double v, double *smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kMcgThreads / 32; ++w) t += smem[w];
  __syncthreads();
  return t;
}

// Warp sum of v (xor shuffle) into smem[warp * K + j]: the first half of
// mcg_block_sum for column j, K columns sharing one barrier.
template <int K>
__device__ __forceinline__ void mcg_warp_slot(double v, int j, double *smemk) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) smemk[(threadIdx.x >> 5) * K + j] = v;
}

// The second half for all K columns: out[j] = the warps' sums in index order
// (threads j < K), then a barrier so smemk can be reused.
template <int K>
__device__ __forceinline__ void mcg_slots_sum(const double *smemk, double *out) {
  __syncthreads();
  if (threadIdx.x < K) {
    double t = 0.0;
    for (int w = 0; w < kMcgThreads / 32; ++w) t += smemk[w * K + threadIdx.x];
    out[threadIdx.x] = t;
  }
  __syncthreads();
}

// K column sums of [K][npart] partials, in index order, into out[K] (shared;
// smemk: K doubles per warp).
template <int K>
__device__ __forceinline__ void mcg_reduce(const double *__restrict__ part, int npart, double *smemk, double *out) {
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = 0.0;
    for (int i = threadIdx.x; i < npart; i += kMcgThreads) s += __ldcg(part + (int64_t)j * npart + i);
    mcg_warp_slot<K>(s, j, smemk);
  }
  mcg_slots_sum<K>(smemk, out);
}

// Thread layout: CPL = K / 2 lanes per row, lane `pr` of a row owning the
// column pair (2 pr, 2 pr + 1) as one 16-byte access, so a gathered row of a
// block is one coalesced K * 8-byte access by CPL lanes and the matrix entry
// (column, value) is a broadcast load among them.  Rows per pass: the grid's
// threads / CPL.
template <int K> struct McgLayout {
  static constexpr int CPL = K / 2;
};

// Per-column partials: thread (row, pr) holds columns 2 pr, 2 pr + 1
// (smemk: K doubles per warp; sums[K] shared).
template <int K>
__device__ __forceinline__ void write_pair_partials(double d0, double d1, double *smemk, double *sums,
                                                    double *__restrict__ part) {
  constexpr int CPL = McgLayout<K>::CPL;
  const int pr = threadIdx.x % CPL;
#pragma unroll
  for (int j = 0; j < K; ++j) mcg_warp_slot<K>((pr == j / 2) ? ((j & 1) ? d1 : d0) : 0.0, j, smemk);
  mcg_slots_sum<K>(smemk, sums);
  if (threadIdx.x < K) part[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = sums[threadIdx.x];
}

__device__ __forceinline__ double2 ld2(const double *p) { return __ldg(reinterpret_cast<const double2 *>(p)); }
__device__ __forceinline__ double2 ld2_rw(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void st2(double *p, double a, double b) {
  *reinterpret_cast<double2 *>(p) = make_double2(a, b);
}

// Kernel A.  src = Z (or R); rz_part [K][npart]; rz_prev [K]; rz_out [K].
template <int K>
__global__ void __launch_bounds__(kMcgThreads, 6) mcg_dir_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                              const int32_t *__restrict__ colIdx,
                                                              const double *__restrict__ val,
                                                              const double *__restrict__ src,
                                                              const double *__restrict__ p_prev,
                                                              double *__restrict__ p, double *__restrict__ q,
                                                              const double *__restrict__ rz_part, int npart,
                                                              const double *__restrict__ rz_prev,
                                                              double *__restrict__ rz_out,
                                                              double *__restrict__ pq_part) {
  constexpr int CPL = McgLayout<K>::CPL;
  __shared__ double smem[kMcgThreads / 32 * K];
  __shared__ double sums[K];
  __shared__ double rz[K];
  mcg_reduce<K>(rz_part, npart, smem, rz);
  if (blockIdx.x == 0 && threadIdx.x < K) rz_out[threadIdx.x] = rz[threadIdx.x];
  const int pr = threadIdx.x % CPL, c0 = 2 * pr;
  const double pv0 = rz_prev[c0], pv1 = rz_prev[c0 + 1];
  const double b0 = (pv0 != 0.0 && isfinite(rz[c0])) ? rz[c0] / pv0 : 0.0;
  const double b1 = (pv1 != 0.0 && isfinite(rz[c0 + 1])) ? rz[c0 + 1] / pv1 : 0.0;
  double d0 = 0.0, d1 = 0.0;
  const int64_t rstride = (int64_t)gridDim.x * (kMcgThreads / CPL);
  for (int64_t i = ((int64_t)blockIdx.x * kMcgThreads + threadIdx.x) / CPL; i < n; i += rstride) {
    double a0 = 0.0, a1 = 0.0;
    const int32_t e = rowPtr[i + 1];
    int32_t k = rowPtr[i];
    for (; k + 1 < e; k += 2) {  // two entries' loads in flight
      const int64_t ca = colIdx[k], cb = colIdx[k + 1];
      const double va = val[k], vb = val[k + 1];
      const double2 sa = ld2(src + ca * K + c0), pa = ld2(p_prev + ca * K + c0);
      const double2 sb = ld2(src + cb * K + c0), pb = ld2(p_prev + cb * K + c0);
      a0 = fma(va, fma(b0, pa.x, sa.x), a0);
      a1 = fma(va, fma(b1, pa.y, sa.y), a1);
      a0 = fma(vb, fma(b0, pb.x, sb.x), a0);
      a1 = fma(vb, fma(b1, pb.y, sb.y), a1);
    }
    if (k < e) {
      const int64_t ca = colIdx[k];
      const double va = val[k];
      const double2 sa = ld2(src + ca * K + c0), pa = ld2(p_prev + ca * K + c0);
      a0 = fma(va, fma(b0, pa.x, sa.x), a0);
      a1 = fma(va, fma(b1, pa.y, sa.y), a1);
    }
    const double2 si = ld2(src + i * K + c0), pi = ld2(p_prev + i * K + c0);
    const double p0 = fma(b0, pi.x, si.x), p1 = fma(b1, pi.y, si.y);
    st2(p + i * K + c0, p0, p1);
    st2(q + i * K + c0, a0, a1);
    d0 += a0 * p0;
    d1 += a1 * p1;
  }
  write_pair_partials<K>(d0, d1, smem, sums, pq_part);
}

// Kernel B.  rz_slot [K] (written by kernel A); dinv null = no preconditioner
// (then z is not written and the r.z partials are the r.r ones).
template <int K>
__global__ void __launch_bounds__(kMcgThreads, K == 4 ? 4 : 0) mcg_update_kernel(int32_t n, const double *__restrict__ pq_part,
                                                                 int npart, const double *__restrict__ rz_slot,
                                                                 double *__restrict__ x, double *__restrict__ r,
                                                                 double *__restrict__ z,
                                                                 const double *__restrict__ p,
                                                                 const double *__restrict__ q,
                                                                 const double *__restrict__ dinv,
                                                                 double *__restrict__ rr_part,
                                                                 double *__restrict__ rz_part) {
  constexpr int CPL = McgLayout<K>::CPL;
  __shared__ double smem[kMcgThreads / 32 * K];
  __shared__ double sums[K];
  __shared__ double pq[K];
  mcg_reduce<K>(pq_part, npart, smem, pq);
  const int pr = threadIdx.x % CPL, c0 = 2 * pr;
  const double rz0 = rz_slot[c0], rz1 = rz_slot[c0 + 1];
  const double al0 = (pq[c0] != 0.0 && rz0 != 0.0 && isfinite(pq[c0])) ? rz0 / pq[c0] : 0.0;
  const double al1 = (pq[c0 + 1] != 0.0 && rz1 != 0.0 && isfinite(pq[c0 + 1])) ? rz1 / pq[c0 + 1] : 0.0;
  double rr0 = 0.0, rr1 = 0.0, z0s = 0.0, z1s = 0.0;
  const int64_t rstride = (int64_t)gridDim.x * (kMcgThreads / CPL);
  for (int64_t i = ((int64_t)blockIdx.x * kMcgThreads + threadIdx.x) / CPL; i < n; i += rstride) {
    const int64_t o = i * K + c0;
    const double2 P = ld2(p + o), Q = ld2(q + o), X = ld2_rw(x + o), R = ld2_rw(r + o);
    const double d = dinv ? __ldg(dinv + i) : 1.0;
    const double x0 = fma(al0, P.x, X.x), x1 = fma(al1, P.y, X.y);
    const double r0 = fma(-al0, Q.x, R.x), r1 = fma(-al1, Q.y, R.y);
    st2(x + o, x0, x1);
    st2(r + o, r0, r1);
    rr0 += r0 * r0;
    rr1 += r1 * r1;
    z0s += r0 * (d * r0);
    z1s += r1 * (d * r1);
    if (dinv) st2(z + o, d * r0, d * r1);
  }
  write_pair_partials<K>(rr0, rr1, smem, sums, rr_part);
  write_pair_partials<K>(z0s, z1s, smem, sums, rz_part);
}

// R = B - A X (and Z = D^{-1} R); partials of r.r, r.z and b.b.
template <int K>
__global__ void __launch_bounds__(kMcgThreads) mcg_residual_kernel(int32_t n, const int32_t *__restrict__ rowPtr,
                                                                   const int32_t *__restrict__ colIdx,
                                                                   const double *__restrict__ val,
                                                                   const double *__restrict__ b,
                                                                   const double *__restrict__ x,
                                                                   double *__restrict__ r, double *__restrict__ z,
                                                                   const double *__restrict__ dinv,
                                                                   double *__restrict__ rr_part,
                                                                   double *__restrict__ rz_part,
                                                                   double *__restrict__ bb_part) {
  constexpr int CPL = McgLayout<K>::CPL;
  __shared__ double smem[kMcgThreads / 32 * K];
  __shared__ double sums[K];
  const int pr = threadIdx.x % CPL, c0 = 2 * pr;
  double rr0 = 0.0, rr1 = 0.0, z0s = 0.0, z1s = 0.0, b0s = 0.0, b1s = 0.0;
  const int64_t rstride = (int64_t)gridDim.x * (kMcgThreads / CPL);
  for (int64_t i = ((int64_t)blockIdx.x * kMcgThreads + threadIdx.x) / CPL; i < n; i += rstride) {
    double a0 = 0.0, a1 = 0.0;
    for (int32_t k = rowPtr[i]; k < rowPtr[i + 1]; ++k) {
      const double2 xr = ld2(x + (int64_t)colIdx[k] * K + c0);
      const double v = val[k];
      a0 = fma(v, xr.x, a0);
      a1 = fma(v, xr.y, a1);
    }
    const int64_t o = i * K + c0;
    const double2 B = ld2(b + o);
    const double d = dinv ? __ldg(dinv + i) : 1.0;
    const double r0 = B.x - a0, r1 = B.y - a1;
    st2(r + o, r0, r1);
    if (dinv) st2(z + o, d * r0, d * r1);
    rr0 += r0 * r0;
    rr1 += r1 * r1;
    z0s += r0 * (d * r0);
    z1s += r1 * (d * r1);
    b0s += B.x * B.x;
    b1s += B.y * B.y;
  }
  write_pair_partials<K>(rr0, rr1, smem, sums, rr_part);
  write_pair_partials<K>(z0s, z1s, smem, sums, rz_part);
  write_pair_partials<K>(b0s, b1s, smem, sums, bb_part);
}

// out[j] = sum of partials j (one CTA).
__global__ void mcg_sum_kernel(const double *__restrict__ part, int npart, int k, double *__restrict__ out) {
  __shared__ double smem[kMcgThreads / 32];
  for (int j = 0; j < k; ++j) {
    double s = 0.0;
    for (int i = threadIdx.x; i < npart; i += kMcgThreads) s += part[(int64_t)j * npart + i];
    s = mcg_block_sum(s, smem);
    if (threadIdx.x == 0) out[j] = s;
  }
}

struct McgBuffers {
  double *X = nullptr, *B = nullptr, *R = nullptr, *Z = nullptr, *P0 = nullptr, *P1 = nullptr, *Q = nullptr;
  double *pq = nullptr, *rr = nullptr, *rz = nullptr, *bb = nullptr, *slots = nullptr, *sums = nullptr;
  void release(cudaStream_t s) {
    for (double *p : {X, B, R, Z, P0, P1, Q, pq, rr, rz, bb, slots, sums}) dfree(p, s);
  }
};

// One group of k <= K columns.
template <int K>
bsp_status mcg_group(const CgPlanView &v, int32_t k, const double *Bu, int64_t ldb, double *Xu, int64_t ldx,
                     double *rel, int32_t *iters_out, bool *conv_out, int64_t *bytes, cudaStream_t s) {
  const int32_t n = v.n;
  // one wave of each kernel: the direction kernel (a gather, capped at 40
  // registers for 6 CTAs/SM) and the streaming update / residual kernels
  // each get their own resident-CTA count; a partial array's length is its
  // writer's grid
  auto wave = [&](auto kern) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMcgThreads, 0) != cudaSuccess || occ < 1) occ = 1;
    return (int)std::max<int64_t>(
        1, std::min<int64_t>(ceil_div((int64_t)n * McgLayout<K>::CPL, kMcgThreads), (int64_t)sm_count() * occ));
  };
  const int grid_d = wave(mcg_dir_kernel<K>), grid = wave(mcg_update_kernel<K>);
  const double *dinv = v.prec_bs == 1 ? static_cast<const double *>(v.minv) : nullptr;
  McgBuffers m;
  const size_t nk = (size_t)n * K;
  bsp_status st = BSP_OK;
  auto fail = [&](bsp_status e) {
    m.release(s);
    return e;
  };
  for (double **p : {&m.X, &m.B, &m.R, &m.P0, &m.P1, &m.Q})
    if ((st = dalloc(p, nk, s)) != BSP_OK) return fail(st);
  if (dinv && (st = dalloc(&m.Z, nk, s)) != BSP_OK) return fail(st);
  if ((st = dalloc(&m.pq, (size_t)K * grid_d, s)) != BSP_OK) return fail(st);
  for (double **p : {&m.rr, &m.rz, &m.bb})
    if ((st = dalloc(p, (size_t)K * grid, s)) != BSP_OK) return fail(st);
  if ((st = dalloc(&m.slots, 2 * K, s)) != BSP_OK || (st = dalloc(&m.sums, 2 * K, s)) != BSP_OK) return fail(st);
  std::vector<double> h(2 * K);
#define MCG_CUDA(call)                                                            \
  do {                                                                            \
    const cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                      \
      set_error(std::string("bsp_cg_solve_multi: " #call " -> ") + cudaGetErrorString(e_)); \
      return fail(BSP_ERR_CUDA);                                                  \
    }                                                                             \
  } while (0)
  // B and X into the padded row-major blocks (padding columns zero)
  if (k < K) {
    MCG_CUDA(cudaMemsetAsync(m.B, 0, nk * sizeof(double), s));
    MCG_CUDA(cudaMemsetAsync(m.X, 0, nk * sizeof(double), s));
  }
  MCG_CUDA(cudaMemcpy2DAsync(m.B, K * sizeof(double), Bu, ldb * sizeof(double), k * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  MCG_CUDA(cudaMemcpy2DAsync(m.X, K * sizeof(double), Xu, ldx * sizeof(double), k * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  MCG_CUDA(cudaMemsetAsync(m.P0, 0, nk * sizeof(double), s));
  MCG_CUDA(cudaMemsetAsync(m.slots, 0, 2 * K * sizeof(double), s));
  double *src = dinv ? m.Z : m.R;
  auto residual = [&]() -> bsp_status {
    mcg_residual_kernel<K><<<grid, kMcgThreads, 0, s>>>(n, v.rowPtr, v.colIdx, v.val, m.B, m.X, m.R, m.Z, dinv,
                                                        m.rr, m.rz, m.bb);
    mcg_sum_kernel<<<1, kMcgThreads, 0, s>>>(m.rr, grid, K, m.sums);
    mcg_sum_kernel<<<1, kMcgThreads, 0, s>>>(m.bb, grid, K, m.sums + K);
    BSP_LAUNCH_CHECK();
    return BSP_OK;
  };
  if ((st = residual()) != BSP_OK) return fail(st);
  MCG_CUDA(cudaMemcpyAsync(h.data(), m.sums, 2 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
  MCG_CUDA(cudaStreamSynchronize(s));
  std::vector<double> bb(h.begin() + K, h.end()), rr(h.begin(), h.begin() + K);
  auto done_all = [&]() {
    for (int j = 0; j < k; ++j)
      if (!(rr[j] <= v.tol * v.tol * bb[j])) return false;
    return true;
  };
  const int64_t mat = (int64_t)v.nnz * 12 + 4 * ((int64_t)n + 1);
  // A: matrix, gathered rows of src and P_prev (counted once), P and Q
  // written; B: P, Q, X, R read, X, R (and Z, D^{-1}) written / read
  const int64_t per_iter = mat + (int64_t)n * K * 8 * (dinv ? 11 : 10) + (dinv ? 8 * (int64_t)n : 0);
  int32_t it = 0;
  bool done = done_all();
  while (!done && it < v.max_iters) {
    for (int c = 0; c < v.check_every; ++c, ++it) {
      double *pp = (it & 1) ? m.P1 : m.P0, *pn = (it & 1) ? m.P0 : m.P1;
      double *slot = m.slots + (it & 1) * K, *prev = m.slots + ((it + 1) & 1) * K;
      mcg_dir_kernel<K><<<grid_d, kMcgThreads, 0, s>>>(n, v.rowPtr, v.colIdx, v.val, src, pp, pn, m.Q, m.rz, grid,
                                                       prev, slot, m.pq);
      mcg_update_kernel<K><<<grid, kMcgThreads, 0, s>>>(n, m.pq, grid_d, slot, m.X, m.R, m.Z, pn, m.Q, dinv, m.rr,
                                                        m.rz);
    }
    mcg_sum_kernel<<<1, kMcgThreads, 0, s>>>(m.rr, grid, K, m.sums);
    BSP_LAUNCH_CHECK();
    MCG_CUDA(cudaMemcpyAsync(h.data(), m.sums, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    MCG_CUDA(cudaStreamSynchronize(s));
    bool nan = false;
    for (int j = 0; j < k; ++j) {
      rr[j] = h[j];
      nan = nan || !(h[j] == h[j]);
    }
    done = done_all() || nan;
  }
  // the true residuals decide
  if ((st = residual()) != BSP_OK) return fail(st);
  MCG_CUDA(cudaMemcpyAsync(h.data(), m.sums, 2 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
  MCG_CUDA(cudaMemcpy2DAsync(Xu, ldx * sizeof(double), m.X, K * sizeof(double), k * sizeof(double), n,
                             cudaMemcpyDeviceToDevice, s));
  MCG_CUDA(cudaStreamSynchronize(s));
#undef MCG_CUDA
  bool conv = true;
  for (int j = 0; j < k; ++j) {
    const double r = h[K + j] > 0 ? std::sqrt(h[j] / h[K + j]) : 0.0;
    if (rel) rel[j] = r;
    conv = conv && r <= v.tol;
  }
  *iters_out = it;
  *conv_out = conv;
  *bytes += (int64_t)it * per_iter + 2 * (mat + (int64_t)n * K * 8 * 3);
  m.release(s);
  return BSP_OK;
}

}  // namespace
}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_cg_solve_multi(bsp_cg_plan P, int32_t k, const double *B, int64_t ldb, double *X,
                                         int64_t ldx, double *rel_residuals, bsp_cg_result *res,
                                         bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P && res && k >= 0 && (k == 0 || (B && X)), "null argument");
  BSP_CHECK_ARG(ldb >= k && ldx >= k, "leading dimension smaller than k");
  CgPlanView v;
  cg_plan_view(P, &v);
  if (v.mixed) BSP_FAIL(BSP_ERR_UNSUPPORTED, "several right-hand sides need an FP64 plan");
  if (v.prec_bs > 1) BSP_FAIL(BSP_ERR_UNSUPPORTED, "several right-hand sides take no or Jacobi preconditioning");
  BSP_CHECK_ARG(((uintptr_t)B | (uintptr_t)X) % 8 == 0, "B and X must be 8-byte aligned");
  cudaStream_t s = as_stream(stream);
  *res = bsp_cg_result{};
  cudaEvent_t e0, e1;
  BSP_CUDA(cudaEventCreate(&e0));
  BSP_CUDA(cudaEventCreate(&e1));
  BSP_CUDA(cudaEventRecord(e0, s));
  int32_t iters = 0;
  bool conv = true;
  int64_t bytes = 0;
  std::vector<double> relv((size_t)k, 0.0);
  for (int32_t j0 = 0; j0 < k; j0 += 8) {
    const int32_t kk = std::min<int32_t>(8, k - j0);
    int32_t it = 0;
    bool c = false;
    double *rel = relv.data() + j0;
    bsp_status st;
    if (kk <= 2)
      st = mcg_group<2>(v, kk, B + j0, ldb, X + j0, ldx, rel, &it, &c, &bytes, s);
    else if (kk <= 4)
      st = mcg_group<4>(v, kk, B + j0, ldb, X + j0, ldx, rel, &it, &c, &bytes, s);
    else
      st = mcg_group<8>(v, kk, B + j0, ldb, X + j0, ldx, rel, &it, &c, &bytes, s);
    if (st != BSP_OK) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return st;
    }
    iters = std::max(iters, it);
    conv = conv && c;
  }
  BSP_CUDA(cudaEventRecord(e1, s));
  BSP_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  res->iterations = iters;
  res->seconds = ms * 1e-3;
  res->converged = conv ? 1 : 0;
  res->bytes_moved = bytes;
  double worst = 0.0;
  for (int32_t j = 0; j < k; ++j) {
    worst = std::max(worst, relv[j]);
    if (rel_residuals) rel_residuals[j] = relv[j];
  }
  res->rel_residual = worst;
  if (!conv) {
    set_error("multi-RHS CG: a column stopped above the tolerance");
    return BSP_ERR_NOT_CONVERGED;
  }
  return BSP_OK;
}
