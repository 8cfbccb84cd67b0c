// Internal helpers shared by every translation unit of libbspmv.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string>

#include "../../include/bsp.h"

namespace bsp {

// Thread-local last-error text behind bsp_last_error().
void set_error(const std::string &msg);
void clear_error();

inline cudaStream_t as_stream(bsp_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

#define BSP_FAIL(code, msg)                                                   \
  do {                                                                        \
    ::bsp::set_error(std::string(__func__) + ": " + (msg));                   \
    return (code);                                                            \
  } while (0)

#define BSP_CHECK_ARG(cond, msg)                                              \
  do {                                                                        \
    if (!(cond)) BSP_FAIL(BSP_ERR_INVALID, msg);                              \
  } while (0)

#define BSP_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      ::bsp::set_error(std::string(__func__) + ": " #call " -> " +            \
                       cudaGetErrorString(e_));                               \
      return BSP_ERR_CUDA;                                                    \
    }                                                                         \
  } while (0)

// Checks (and clears) the launch error of the kernel just issued
// (configuration errors only; the kernel itself runs asynchronously).
#define BSP_LAUNCH_CHECK() BSP_CUDA(cudaGetLastError())

#define BSP_TRY(expr)                                                         \
  do {                                                                        \
    bsp_status st_ = (expr);                                                  \
    if (st_ != BSP_OK) return st_;                                            \
  } while (0)

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;  // B200

inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = kNumSMs;
  }
  return n;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Stream-ordered device allocation (cudaMallocAsync pool).
template <typename T>
bsp_status dalloc(T **p, size_t count, cudaStream_t s) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(p), count * sizeof(T), s);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMallocAsync(") + std::to_string(count * sizeof(T)) +
              " B) -> " + cudaGetErrorString(e));
    return BSP_ERR_ALLOC;
  }
  return BSP_OK;
}

template <typename T>
void dfree(T *&p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
  p = nullptr;
}

// ---------------------------------------------------------------------------
// Device-side load helpers.  Streamed matrix data is read once: bypass L1 and
// mark it evict-first in L2 so the gathered vector x stays resident.  sm_100
// has 256-bit global loads; they take the eviction qualifier directly.
struct f64x4 {
  double x, y, z, w;
};
__device__ __forceinline__ f64x4 ld_stream_f64x4(const double *p) {
  f64x4 r;
  asm("ld.global.nc.L1::no_allocate.L2::evict_first.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
               : "l"(p));
  return r;
}
// Same with a 256-byte L2 fetch granularity hint for long sequential streams.
__device__ __forceinline__ f64x4 ld_stream_f64x4_pf(const double *p) {
  f64x4 r;
  asm("ld.global.nc.L1::no_allocate.L2::evict_first.L2::256B.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w)
      : "l"(p));
  return r;
}
// 256-bit read-only load with default caching (x gathers: keep in L2/L1).
__device__ __forceinline__ f64x4 ld_x4(const double *p) {
  f64x4 r;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double2 ld_stream_f64x2(const double *p, uint64_t pol) {
  double2 r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
               : "=d"(r.x), "=d"(r.y)
               : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ double ld_stream_f64(const double *p, uint64_t pol) {
  double r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ int ld_stream_s32(const int *p, uint64_t pol) {
  int r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
  return r;
}
// Gathers of x: read-only path, default caching.
__device__ __forceinline__ double ld_x(const double *p) { return __ldg(p); }

__device__ __forceinline__ double2 ld_x2(const double *p) {
  return __ldg(reinterpret_cast<const double2 *>(p));
}

__device__ __forceinline__ void st_stream_f64(double *p, double v) {
  asm volatile("st.global.cs.f64 [%0], %1;" ::"l"(p), "d"(v));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v, unsigned mask = 0xffffffffu) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

}  // namespace bsp

// What the multi-right-hand-side CG (cg_multi.cu) reads from a CG plan (cg.cu).
struct bsp_cg_plan_s;
namespace bsp {
struct CgPlanView {
  int32_t n, nnz;
  const int32_t *rowPtr, *colIdx;
  const double *val;
  bool mixed;
  int prec_bs;
  const void *minv;
  int32_t check_every, max_iters;
  double tol;
};
void cg_plan_view(const bsp_cg_plan_s *P, CgPlanView *v);
}  // namespace bsp
