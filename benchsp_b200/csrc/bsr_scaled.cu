// BSR with FP16/BF16 values and one power-of-two scale per block.
//
// The FP64 BSR SpMV reads 132 bytes per 4x4 block (128 of values, 4 of block
// column); it runs at the HBM copy rate, so the only way to go faster is to
// move fewer bytes.  Here a block keeps its 16 values as 16-bit floats (32
// bytes) and one exponent packed with its block column into a 32-bit key:
// 36 bytes per block, 3.7x fewer.  The exponent keeps every block inside the
// 16-bit type's normal range whatever the matrix's overall scale.
//
// SpMV mapping: one lane per 4x4 tile (a whole 4x4 block, or a quarter of an
// 8x8 block): one 256-bit streaming load of the tile, one 4-byte key load,
// one 4-entry load of x.  x is rounded to FP32 and scaled by the block's 2^e
// (exact), then 16 FP32 FMAs into 4 row accumulators; LG lanes share a block
// row and reduce with shuffles at the end.
#include "bsp_internal.cuh"

namespace bsp {

constexpr int kScaledBias = 128;
constexpr uint32_t kScaledColMask = 0x00FFFFFFu;

__device__ __forceinline__ float2 lp2_to_f32(uint32_t u, int dt) {
  if (dt == BSP_BF16) return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xFFFF0000u));
  __half2 h;
  memcpy(&h, &u, 4);
  return __half22float2(h);
}

// 2^e as a float, e in [-126, 127].
__device__ __forceinline__ float pow2f(int e) { return __uint_as_float((uint32_t)(e + 127) << 23); }

// ---------------------------------------------------------------------------
// Conversion: one thread per block.

template <int BS, int DT>
__global__ void bsr_scale_kernel(int64_t nb, const int32_t *__restrict__ blcIdx, const double *__restrict__ blcVal,
                                 uint32_t *__restrict__ key, uint16_t *__restrict__ out, int32_t *__restrict__ bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const double *v = blcVal + k * (BS * BS);
  double m = 0.0;
  bool finite = true;
  for (int i = 0; i < BS * BS; ++i) {
    const double a = fabs(v[i]);
    finite = finite && (a <= 1.7976931348623157e308);   // false for inf and NaN
    m = fmax(m, a);
  }
  int e = 0;
  if (m > 0.0) {
    const int E = (int)((__double_as_longlong(m) >> 52) & 0x7FF) - 1023;  // floor(log2 m); -1023 if subnormal
    e = DT == BSP_F16 ? E - 14 : E;
    e = max(-126, min(127, e));
  }
  const double down = __longlong_as_double((long long)(1023 - e) << 52);   // 2^-e, exact
  bool ok = finite;
  uint16_t *o = out + k * (BS * BS);
  for (int r = 0; r < BS; ++r)
    for (int c = 0; c < BS; ++c) {
      const float f = __double2float_rn(v[r * BS + c] * down);
      uint16_t q;
      if (DT == BSP_F16) {
        const __half h = __float2half_rn(f);
        q = __half_as_ushort(h);
        ok = ok && ((q & 0x7C00u) != 0x7C00u);   // not inf / NaN
      } else {
        const __nv_bfloat16 b = __float2bfloat16_rn(f);
        q = __bfloat16_as_ushort(b);
        ok = ok && ((q & 0x7F80u) != 0x7F80u);
      }
      // tile (r/4, c/4), entry (r%4, c%4) inside the tile
      const int t = (r >> 2) * (BS / 4) + (c >> 2);
      o[t * 16 + (r & 3) * 4 + (c & 3)] = q;
    }
  key[k] = (uint32_t)blcIdx[k] | ((uint32_t)(e + kScaledBias) << 24);
  if (!ok) atomicExch(bad, 1);
}

// ---------------------------------------------------------------------------
// SpMV.  BS = 4 or 8; DT = BSP_F16 / BSP_BF16; LG lanes per block row; U
// blocks per lane per loop trip; XT/YT = double or float; XV = x may be read
// 4 entries at a time (aligned).

template <typename XT>
__device__ __forceinline__ float4 ld_x4f(const XT *p, int64_t xc, int32_t col, bool vec) {
  if (vec && xc + 4 <= col) {
    if constexpr (sizeof(XT) == 8) {
      const f64x4 v = ld_x4(reinterpret_cast<const double *>(p + xc));
      return make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
    } else {
      return __ldg(reinterpret_cast<const float4 *>(p + xc));
    }
  }
  float4 r;
  r.x = xc < col ? (float)__ldg(p + xc) : 0.f;
  r.y = xc + 1 < col ? (float)__ldg(p + xc + 1) : 0.f;
  r.z = xc + 2 < col ? (float)__ldg(p + xc + 2) : 0.f;
  r.w = xc + 3 < col ? (float)__ldg(p + xc + 3) : 0.f;
  return r;
}

template <int BS, int DT, int LG, int U, typename XT, typename YT, bool XV>
__global__ void __launch_bounds__(256) bsr_scaled_kernel(int32_t blc_row, int32_t row, int32_t col,
                                                         const int32_t *__restrict__ blcPtr,
                                                         const uint32_t *__restrict__ blcKey,
                                                         const uint16_t *__restrict__ blcVal,
                                                         const XT *__restrict__ x, YT *__restrict__ y,
                                                         double alpha, double beta) {
  constexpr int TS = BS / 4;          // tiles per block side
  constexpr int TPB = TS * TS;        // lanes per block
  constexpr int BPS = LG / TPB;       // blocks per group step
  static_assert(LG % TPB == 0 && LG <= 32, "bad lane group");
  const int lane = threadIdx.x & 31;
  const int gl = lane & (LG - 1);
  const int slot = gl / TPB;
  const int t = gl % TPB;
  const int tr = t / TS, tc = t % TS;
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / LG);
  const int64_t warp_first = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LG;
  for (int64_t base = warp_first; base < blc_row; base += groups) {
    const int64_t br = base + lane / LG;
    const bool active = br < blc_row;
    const int32_t s = active ? blcPtr[br] : 0;
    const int32_t e = active ? blcPtr[br + 1] : 0;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    // 4x4 blocks: the next trip's keys are loaded before this trip's x
    // gathers, so a trip waits on one round trip (x) instead of two (key,
    // then x): stencil 64^3 x 4 dof, FP16, FP64 x / y 47.9 -> 44.0 us.  For
    // 8x8 blocks it measured 66.9 -> 72.3 us with FP32 x / y and stays off.
    constexpr bool PF = BS == 4;
    uint32_t kcur[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int32_t k = s + slot + u * BPS;
      kcur[u] = (PF && k < e) ? __ldg(blcKey + k) : 0u;
    }
    for (int32_t k0 = s + slot; k0 < e; k0 += BPS * U) {
      f64x4 raw[U];
      float4 xv[U];
      uint32_t knext[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t kn = k0 + BPS * U + u * BPS;
        knext[u] = (PF && kn < e) ? __ldg(blcKey + kn) : 0u;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t k = k0 + u * BPS;
        if (k < e) {
          raw[u] = ld_stream_f64x4(reinterpret_cast<const double *>(blcVal + (int64_t)k * (BS * BS) + 16 * t));
          const uint32_t key = PF ? kcur[u] : __ldg(blcKey + k);
          const int64_t xc = (int64_t)(key & kScaledColMask) * BS + 4 * tc;
          xv[u] = ld_x4f<XT>(x, xc, col, XV);
          const float sc = pow2f((int)(key >> 24) - kScaledBias);
          xv[u].x *= sc;
          xv[u].y *= sc;
          xv[u].z *= sc;
          xv[u].w *= sc;
        } else {
          raw[u] = f64x4{0.0, 0.0, 0.0, 0.0};
          xv[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) kcur[u] = knext[u];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const double w[4] = {raw[u].x, raw[u].y, raw[u].z, raw[u].w};
        float acc[4] = {a0, a1, a2, a3};
#pragma unroll
        for (int i = 0; i < 4; ++i) {   // tile row i: 4 values in one 64-bit word
          const uint64_t bits = (uint64_t)__double_as_longlong(w[i]);
          const float2 q01 = lp2_to_f32((uint32_t)bits, DT);
          const float2 q23 = lp2_to_f32((uint32_t)(bits >> 32), DT);
          float s0 = acc[i];
          s0 = fmaf(q01.x, xv[u].x, s0);
          s0 = fmaf(q01.y, xv[u].y, s0);
          s0 = fmaf(q23.x, xv[u].z, s0);
          s0 = fmaf(q23.y, xv[u].w, s0);
          acc[i] = s0;
        }
        a0 = acc[0];
        a1 = acc[1];
        a2 = acc[2];
        a3 = acc[3];
      }
    }
    // Sum over the lanes of the group that hold the same tile row: every
    // lane bit except the tile-row bit (bit log2(TS) of t when TS = 2).
#pragma unroll
    for (int o = 1; o < LG; o <<= 1) {
      if (TS == 2 && o == 2) continue;
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      a3 += __shfl_xor_sync(0xffffffffu, a3, o);
    }
    if (active && slot == 0 && tc == 0) {
      const int64_t y0 = br * BS + 4 * tr;
      const float acc[4] = {a0, a1, a2, a3};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int64_t yi = y0 + i;
        if (yi < row) {
          double res = alpha * (double)acc[i];
          if (beta != 0.0) res += beta * (double)y[yi];
          y[yi] = (YT)res;
        }
      }
    }
  }
}

using ScaledLauncher = void (*)(const bsp_bsr_scaled *, const void *, void *, double, double, bool, cudaStream_t);

template <int BS, int DT, int LG, int U, typename XT, typename YT>
static void launch_scaled(const bsp_bsr_scaled *m, const void *x, void *y, double a, double b, bool xv,
                          cudaStream_t s) {
  int64_t blocks = ceil_div(m->blc_row, 256 / LG);
  const int64_t cap = (int64_t)sm_count() * 64;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  const XT *xp = static_cast<const XT *>(x);
  YT *yp = static_cast<YT *>(y);
  if (xv)
    bsr_scaled_kernel<BS, DT, LG, U, XT, YT, true><<<(unsigned)blocks, 256, 0, s>>>(
        m->blc_row, m->row, m->col, m->blcPtr, m->blcKey, m->blcVal, xp, yp, a, b);
  else
    bsr_scaled_kernel<BS, DT, LG, U, XT, YT, false><<<(unsigned)blocks, 256, 0, s>>>(
        m->blc_row, m->row, m->col, m->blcPtr, m->blcKey, m->blcVal, xp, yp, a, b);
}

struct ScaledVariant {
  int bs, dt, lanes, unroll, xdt, ydt;
  ScaledLauncher fn;
};

#define BSP_SV_T(BS, DT, LG, U)                                                                   \
  {BS, DT, LG, U, BSP_F64, BSP_F64, &launch_scaled<BS, DT, LG, U, double, double>},               \
      {BS, DT, LG, U, BSP_F32, BSP_F64, &launch_scaled<BS, DT, LG, U, float, double>},            \
      {BS, DT, LG, U, BSP_F64, BSP_F32, &launch_scaled<BS, DT, LG, U, double, float>},            \
      {BS, DT, LG, U, BSP_F32, BSP_F32, &launch_scaled<BS, DT, LG, U, float, float>}
#define BSP_SV(BS, LG, U) BSP_SV_T(BS, BSP_F16, LG, U), BSP_SV_T(BS, BSP_BF16, LG, U)

static const ScaledVariant kScaledVariants[] = {
    BSP_SV(4, 4, 1),  BSP_SV(4, 8, 1),  BSP_SV(4, 16, 1),  BSP_SV(4, 32, 1), BSP_SV(4, 4, 2),
    BSP_SV(4, 8, 2),  BSP_SV(4, 16, 2), BSP_SV(8, 4, 1),   BSP_SV(8, 8, 1),  BSP_SV(8, 16, 1),
    BSP_SV(8, 32, 1), BSP_SV(8, 8, 2),  BSP_SV(8, 16, 2),
};
#undef BSP_SV
#undef BSP_SV_T

static const ScaledVariant *find_scaled(int bs, int dt, int lanes, int unroll, int xdt, int ydt) {
  for (const ScaledVariant &v : kScaledVariants)
    if (v.bs == bs && v.dt == dt && v.lanes == lanes && v.unroll == unroll && v.xdt == xdt && v.ydt == ydt)
      return &v;
  return nullptr;
}

// Default shape, one block per trip: a lane walks about 6-8 blocks of its
// block row for 4x4 blocks and about 3-4 tiles for 8x8 blocks.  Measured on
// the 27-point stencil 64^3 x 4 dof (27 blocks per block row), FP16: 4x4 at
// 4 lanes 47.9 us, 8 lanes 48.3, 16 lanes 53.8, 32 lanes 66.2; 8x8 (14.3
// blocks per block row) at 16 lanes 76.6 us, 8 lanes 78.6, 32 lanes 82.6.
static void default_shape(const bsp_bsr_scaled *m, int *lanes, int *unroll) {
  const double avg = m->blc_row > 0 ? (double)m->blc_num / (double)m->blc_row : 0.0;
  const int tpb = (m->bs / 4) * (m->bs / 4);
  const double per_lane = m->bs == 4 ? 6.0 : 3.5;
  int lg = 4;
  while (lg < 32 && avg * tpb > per_lane * 2 * lg) lg <<= 1;
  if (lg < tpb) lg = tpb;
  *lanes = lg;
  *unroll = 1;
}

static bsp_status scaled_spmv(const bsp_bsr_scaled *m, const void *x, int32_t xdt, void *y, int32_t ydt, double a,
                              double b, int lanes, int unroll, cudaStream_t s) {
  BSP_CHECK_ARG(m && x && y, "null pointer");
  BSP_CHECK_ARG(m->bs == 4 || m->bs == 8, "block size must be 4 or 8");
  BSP_CHECK_ARG(m->dtype == BSP_F16 || m->dtype == BSP_BF16, "matrix dtype must be BSP_F16 or BSP_BF16");
  BSP_CHECK_ARG((xdt == BSP_F64 || xdt == BSP_F32) && (ydt == BSP_F64 || ydt == BSP_F32),
                "x and y must be BSP_F64 or BSP_F32");
  if (m->blc_row == 0) return BSP_OK;
  if (((uintptr_t)m->blcVal & 31) != 0) BSP_FAIL(BSP_ERR_INVALID, "blcVal must be 32-byte aligned");
  if (lanes == 0) default_shape(m, &lanes, &unroll);
  const ScaledVariant *v = find_scaled(m->bs, m->dtype, lanes, unroll, xdt, ydt);
  if (!v) BSP_FAIL(BSP_ERR_UNSUPPORTED, "no scaled BSR kernel with these lanes/unroll");
  const size_t xa = xdt == BSP_F64 ? 32 : 16;   // one 4-entry load
  const bool xv = ((uintptr_t)x % xa) == 0;
  v->fn(m, x, y, a, b, xv, s);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_bsr_scaled_create(const bsp_bsr *src, int32_t dtype, bsp_bsr_scaled *out,
                                            bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(src && out, "null pointer");
  BSP_CHECK_ARG(src->bs == 4 || src->bs == 8, "block size must be 4 or 8");
  BSP_CHECK_ARG(dtype == BSP_F16 || dtype == BSP_BF16, "dtype must be BSP_F16 or BSP_BF16");
  BSP_CHECK_ARG(src->blc_num >= 0 && src->blc_row >= 0, "malformed BSR descriptor");
  if (src->blc_col >= (1 << 24))
    BSP_FAIL(BSP_ERR_UNSUPPORTED, "the scaled format holds block columns below 2^24");
  cudaStream_t s = as_stream(stream);
  bsp_bsr_scaled m{};
  m.row = src->row;
  m.col = src->col;
  m.bs = src->bs;
  m.blc_row = src->blc_row;
  m.blc_col = src->blc_col;
  m.blc_num = src->blc_num;
  m.dtype = dtype;
  const size_t nb = (size_t)src->blc_num;
  const int bb = src->bs * src->bs;
  int32_t *bad = nullptr;
  bsp_status st = dalloc(&m.blcPtr, (size_t)src->blc_row + 1, s);
  if (st == BSP_OK) st = dalloc(&m.blcKey, nb, s);
  if (st == BSP_OK) st = dalloc(&m.blcVal, nb * bb, s);
  if (st == BSP_OK) st = dalloc(&bad, 1, s);
  cudaError_t e = cudaSuccess;
  if (st == BSP_OK) {
    e = cudaMemcpyAsync(m.blcPtr, src->blcPtr, sizeof(int32_t) * ((size_t)src->blc_row + 1),
                        cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
    if (e == cudaSuccess && nb > 0) {
      const unsigned grid = (unsigned)ceil_div((int64_t)nb, 256);
      if (src->bs == 4 && dtype == BSP_F16)
        bsr_scale_kernel<4, BSP_F16><<<grid, 256, 0, s>>>(nb, src->blcIdx, src->blcVal, m.blcKey, m.blcVal, bad);
      else if (src->bs == 4)
        bsr_scale_kernel<4, BSP_BF16><<<grid, 256, 0, s>>>(nb, src->blcIdx, src->blcVal, m.blcKey, m.blcVal, bad);
      else if (dtype == BSP_F16)
        bsr_scale_kernel<8, BSP_F16><<<grid, 256, 0, s>>>(nb, src->blcIdx, src->blcVal, m.blcKey, m.blcVal, bad);
      else
        bsr_scale_kernel<8, BSP_BF16><<<grid, 256, 0, s>>>(nb, src->blcIdx, src->blcVal, m.blcKey, m.blcVal, bad);
      e = cudaGetLastError();
    }
  }
  int32_t hbad = 0;
  if (st == BSP_OK && e == cudaSuccess) {
    e = cudaMemcpyAsync(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  dfree(bad, s);
  if (st == BSP_OK && e != cudaSuccess) {
    set_error(std::string("bsp_bsr_scaled_create: ") + cudaGetErrorString(e));
    st = BSP_ERR_CUDA;
  }
  if (st == BSP_OK && hbad) {
    set_error("bsp_bsr_scaled_create: a value is not finite or its block overflows the 16-bit type");
    st = BSP_ERR_INVALID;
  }
  if (st != BSP_OK) {
    dfree(m.blcPtr, s);
    dfree(m.blcKey, s);
    dfree(m.blcVal, s);
    cudaStreamSynchronize(s);
    return st;
  }
  *out = m;
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_scaled_free(bsp_bsr_scaled *m) {
  clear_error();
  if (!m) return BSP_OK;
  cudaStream_t s = 0;
  dfree(m->blcPtr, s);
  dfree(m->blcKey, s);
  dfree(m->blcVal, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_scaled_spmv(const bsp_bsr_scaled *m, const void *x, int32_t x_dtype, void *y,
                                          int32_t y_dtype, double alpha, double beta, bsp_stream_t stream) {
  clear_error();
  return scaled_spmv(m, x, x_dtype, y, y_dtype, alpha, beta, 0, 0, as_stream(stream));
}

extern "C" bsp_status bsp_bsr_scaled_spmv_variant(const bsp_bsr_scaled *m, const void *x, int32_t x_dtype,
                                                  void *y, int32_t y_dtype, double alpha, double beta,
                                                  int32_t lanes_per_blockrow, int32_t unroll, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(lanes_per_blockrow > 0 && (unroll == 1 || unroll == 2), "lanes must be > 0 and unroll 1 or 2");
  return scaled_spmv(m, x, x_dtype, y, y_dtype, alpha, beta, lanes_per_blockrow, unroll, as_stream(stream));
}
