// SpMM C = alpha*A*B + beta*C with A sparse, B and C dense row-major.
//
// Replaces the reference's SMaT-style FP16 SpMM (mmaSmatKernelfp16 /
// smatSpmmfp16, src/smat.cu:22-201): one warp per 16x8 C tile, a 16x16 A
// block and a 16x8 B tile copied to shared memory, ldmatrix and
// mma.sync m16n8k16 with FP16 accumulation.  (It also divides an already
// block-level column index by 16 again, smat.cu:49, addresses B correctly
// only for K = 16, smat.cu:62-64, and never writes its output.)  Two paths:
//
//  * CSR SpMM (any sparsity): one warp per row; the row's column indices and
//    values are loaded 32 at a time and broadcast by shuffle; every lane owns
//    CPL consecutive columns of B/C and streams its slice of each gathered B
//    row with one vector load; FP32 accumulation, FP32 C.
//  * Block SpMM (16x16 tiles, for matrices whose tiles are dense): one warp
//    per (block-row, 8*NT columns).  Lane 0 stages every A tile (512 B) and
//    the 16 matching B row segments with cp.async.bulk (the TMA copy engine)
//    into a STAGES-deep shared-memory ring completed on mbarriers; the warp
//    reads fragments with ldmatrix (.trans for B) and issues
//    mma.sync.m16n8k16 with FP32 accumulators.  Every wait is bounded: on
//    timeout the kernel records an error, waits (bounded) for its own copies
//    and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

template <typename T> __device__ __forceinline__ float sp_to_float(T v);
template <> __device__ __forceinline__ float sp_to_float<float>(float v) { return v; }
template <> __device__ __forceinline__ float sp_to_float<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float sp_to_float<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// CPL consecutive elements of type T as one vector load.
template <typename T, int CPL>
__device__ __forceinline__ void load_cols(const T *p, float (&out)[CPL]) {
  constexpr int BYTES = CPL * (int)sizeof(T);
  if constexpr (BYTES == 16) {
    const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
    const T *t = reinterpret_cast<const T *>(&u);
#pragma unroll
    for (int k = 0; k < CPL; ++k) out[k] = sp_to_float<T>(t[k]);
  } else if constexpr (BYTES == 8) {
    const uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
    const T *t = reinterpret_cast<const T *>(&u);
#pragma unroll
    for (int k = 0; k < CPL; ++k) out[k] = sp_to_float<T>(t[k]);
  } else if constexpr (BYTES == 4) {
    const unsigned u = __ldg(reinterpret_cast<const unsigned *>(p));
    const T *t = reinterpret_cast<const T *>(&u);
#pragma unroll
    for (int k = 0; k < CPL; ++k) out[k] = sp_to_float<T>(t[k]);
  } else {
#pragma unroll
    for (int k = 0; k < CPL; ++k) out[k] = sp_to_float<T>(p[k]);
  }
}

// Warp per row; lane owns columns c0 + lane*CPL .. +CPL of each 32*CPL chunk.
template <typename T, int CPL>
__global__ void __launch_bounds__(256) spmm_csr_kernel(int32_t rows, int32_t N, const int32_t *__restrict__ rowPtr,
                                                       const int32_t *__restrict__ colIdx,
                                                       const T *__restrict__ val, const T *__restrict__ B,
                                                       int64_t ldb, float *__restrict__ C, int64_t ldc,
                                                       float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nwarps) {
    const int32_t s = rowPtr[r], e = rowPtr[r + 1];
    for (int32_t c0 = 0; c0 < N; c0 += 32 * CPL) {
      const int32_t cl = c0 + lane * CPL;
      const bool own = cl < N;  // N is a multiple of CPL
      float acc[CPL];
#pragma unroll
      for (int k = 0; k < CPL; ++k) acc[k] = 0.f;
      for (int32_t j0 = s; j0 < e; j0 += 32) {
        const int32_t j = j0 + lane;
        const int32_t cj = j < e ? colIdx[j] : 0;
        const float vj = j < e ? sp_to_float<T>(val[j]) : 0.f;
        const int cnt = e - j0 < 32 ? e - j0 : 32;
        int t = 0;
        for (; t + 4 <= cnt; t += 4) {  // four B rows in flight
          float b[4][CPL];
          float v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int32_t c = __shfl_sync(0xffffffffu, cj, t + u);
            v[u] = __shfl_sync(0xffffffffu, vj, t + u);
            if (own) load_cols<T, CPL>(B + (int64_t)c * ldb + cl, b[u]);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < CPL; ++k) acc[k] = fmaf(v[u], b[u][k], acc[k]);
        }
        for (; t < cnt; ++t) {
          const int32_t c = __shfl_sync(0xffffffffu, cj, t);
          const float v = __shfl_sync(0xffffffffu, vj, t);
          float b[CPL];
          if (own) {
            load_cols<T, CPL>(B + (int64_t)c * ldb + cl, b);
#pragma unroll
            for (int k = 0; k < CPL; ++k) acc[k] = fmaf(v, b[k], acc[k]);
          }
        }
      }
      if (own) {
        float *cp = C + r * ldc + cl;
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
          float o = alpha * acc[k];
          if (beta != 0.f) o += beta * cp[k];
          cp[k] = o;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Grouped CSR SpMM engine.  Every lane moves 16 bytes (VEC elements) of a
// gathered B row; LPR lanes cover LPR*VEC columns of one row, so one warp step
// handles G = 32/LPR nonzeros at once (N = 32 FP16: 8 nonzeros of 64 bytes
// each), and kSpmmU steps are in flight.  The row's 32 column indices and
// values are loaded once per chunk of 32 and broadcast by shuffle.  After the
// segment the G groups' partial sums are added with a fixed shuffle tree, so
// every lane holds the totals (deterministic).
constexpr int kSpmmU = 4;

template <typename T> struct SpmmVec { static constexpr int VEC = 16 / (int)sizeof(T); };

template <typename T>
__device__ __forceinline__ void unpack16(const uint4 &u, float (&o)[SpmmVec<T>::VEC]);
template <>
__device__ __forceinline__ void unpack16<float>(const uint4 &u, float (&o)[4]) {
  o[0] = __uint_as_float(u.x);
  o[1] = __uint_as_float(u.y);
  o[2] = __uint_as_float(u.z);
  o[3] = __uint_as_float(u.w);
}
template <>
__device__ __forceinline__ void unpack16<__half>(const uint4 &u, float (&o)[8]) {
  const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __half2 h;
    memcpy(&h, &w[k], 4);
    const float2 f = __half22float2(h);
    o[2 * k] = f.x;
    o[2 * k + 1] = f.y;
  }
}
template <>
__device__ __forceinline__ void unpack16<__nv_bfloat16>(const uint4 &u, float (&o)[8]) {
  const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __nv_bfloat162 h;
    memcpy(&h, &w[k], 4);
    const float2 f = __bfloat1622float2(h);
    o[2 * k] = f.x;
    o[2 * k + 1] = f.y;
  }
}

// acc (this lane's VEC columns starting at cl) += sum over nonzeros [s, e).
template <typename T, int LPR>
__device__ __forceinline__ void spmm_segment(int32_t s, int32_t e, const int32_t *__restrict__ colIdx,
                                             const T *__restrict__ val, const T *__restrict__ B, int64_t ldb,
                                             int32_t cl, int lane, float (&acc)[SpmmVec<T>::VEC]) {
  constexpr int VEC = SpmmVec<T>::VEC;
  constexpr int G = 32 / LPR;
  const int g = lane / LPR;
  for (int32_t j0 = s; j0 < e; j0 += 32) {
    const int32_t j = j0 + lane;
    const int32_t cj = j < e ? __ldg(colIdx + j) : 0;
    const float vj = j < e ? sp_to_float<T>(__ldg(val + j)) : 0.f;
    const int cnt = e - j0 < 32 ? e - j0 : 32;
    for (int t = 0; t < cnt; t += G * kSpmmU) {  // warp-uniform bounds
      uint4 raw[kSpmmU];
      float v[kSpmmU];
#pragma unroll
      for (int u = 0; u < kSpmmU; ++u) {
        const int src = t + u * G + g;
        const int32_t c = __shfl_sync(0xffffffffu, cj, src & 31);
        const float vv = __shfl_sync(0xffffffffu, vj, src & 31);
        const bool ok = src < cnt;
        v[u] = ok ? vv : 0.f;
        raw[u] = ok ? __ldg(reinterpret_cast<const uint4 *>(B + (int64_t)c * ldb + cl)) : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int u = 0; u < kSpmmU; ++u) {
        float b[VEC];
        unpack16<T>(raw[u], b);
#pragma unroll
        for (int k = 0; k < VEC; ++k) acc[k] = fmaf(v[u], b[k], acc[k]);
      }
    }
  }
#pragma unroll
  for (int o = LPR; o < 32; o <<= 1)
#pragma unroll
    for (int k = 0; k < VEC; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
}

// Warp per row; column passes of LPR*VEC columns.
// Wide B rows (8+ lanes per row, N >= 64 in FP16) are gather-latency bound:
// capping registers at 40 keeps 6 CTAs per SM resident instead of 4 (graph
// 2^20, FP16: N = 128 2.43 -> 2.16 ms, N = 256 4.43 -> 3.99 ms); narrow rows
// lose 1% with the cap and keep the compiler's default (a minimum of 0 CTAs
// leaves the register choice unconstrained, like no second bound; an explicit
// 1 would let it take more registers than the default).
template <typename T, int LPR>
__global__ void __launch_bounds__(256, LPR >= 8 ? 6 : 0) spmm_grouped_kernel(int32_t rows, int32_t N, const int32_t *__restrict__ rowPtr,
                                                           const int32_t *__restrict__ colIdx,
                                                           const T *__restrict__ val, const T *__restrict__ B,
                                                           int64_t ldb, float *__restrict__ C, int64_t ldc,
                                                           float alpha, float beta) {
  constexpr int VEC = SpmmVec<T>::VEC;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nwarps) {
    const int32_t s = rowPtr[r], e = rowPtr[r + 1];
    for (int32_t c0 = 0; c0 < N; c0 += LPR * VEC) {
      const int32_t cl = c0 + (lane % LPR) * VEC;
      float acc[VEC];
#pragma unroll
      for (int k = 0; k < VEC; ++k) acc[k] = 0.f;
      spmm_segment<T, LPR>(s, e, colIdx, val, B, ldb, cl, lane, acc);
      if (lane < LPR) {
        float *cp = C + r * ldc + cl;
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          float o = alpha * acc[k];
          if (beta != 0.f) o += beta * cp[k];
          cp[k] = o;
        }
      }
    }
  }
}

// Lanes per B row for the grouped kernels: the largest power of two <= 32
// with LPR * VEC dividing N; 0 when B's rows are not 16-byte aligned or N is
// not a multiple of VEC (then the scalar-column kernels run).
template <typename T>
static int grouped_lpr(int32_t N, const void *B, int64_t ldb) {
  constexpr int VEC = SpmmVec<T>::VEC;
  if ((uintptr_t)B % 16 != 0 || (ldb * (int64_t)sizeof(T)) % 16 != 0 || N % VEC != 0) return 0;
  int l = 32;
  while (l > 1 && (N % (l * VEC) != 0)) l >>= 1;
  return l;
}

// Position of tile element (row n, column k) in the stored tile: four 8x8
// core matrices of 128 contiguous bytes, core (n/8, k/8) at (2*(n/8) + k/8)
// * 64 elements, row n%8 of it at 8*(n%8).  This is the no-swizzle K-major
// operand layout of tcgen05.mma (rows 16 bytes apart inside a core matrix,
// K halves 128 bytes apart, 8-row groups 256 bytes apart); ldmatrix reads
// the same 16-byte rows.
__host__ __device__ __forceinline__ int tile_pos(int n, int k) {
  return ((n >> 3) * 2 + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7);
}

// ---------------------------------------------------------------------------
// Block (16x16) tensor-core SpMM.
constexpr int kTS = 16;            // tile side
constexpr int kStages = 4;         // shared-memory ring depth per warp
constexpr int kWarpsPerCta = 4;
constexpr long long kSpinLimit = 1ll << 24;  // bounded mbarrier waits

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// alpha * acc + beta * c with a fixed rounding (one product, one fused
// multiply-add) so that every tensor-core kernel stores the same bits for the
// same accumulator, whatever contraction the compiler would choose.
__device__ __forceinline__ float scale_out(float alpha, float acc, float beta, const float *cp) {
  const float o = __fmul_rn(alpha, acc);
  return beta != 0.f ? __fmaf_rn(beta, *cp, o) : o;
}
// Bounded wait; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void ldm_x4(uint32_t (&r)[4], const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldm_x4_trans(uint32_t (&r)[4], const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
template <typename T>
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1);
template <>
__device__ __forceinline__ void mma16816<__half>(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
template <>
__device__ __forceinline__ void mma16816<__nv_bfloat16>(float (&c)[4], const uint32_t (&a)[4], uint32_t b0,
                                                        uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Per-warp ring slot: A tile (16x16) then B rows (16 x 8*NT) at a padded
// row stride so the 8 rows an ldmatrix reads fall in different banks.
template <int NT>
struct SpmmStage {
  static constexpr int kBStride = 8 * NT * 2 + 16;  // bytes per staged B row
  alignas(128) unsigned char a[kTS * kTS * 2];
  alignas(16) unsigned char b[kTS * kBStride];
};

template <typename T, int NT>
__global__ void __launch_bounds__(kWarpsPerCta * 32) spmm_block_kernel(
    int32_t M, int32_t K, int32_t N, int32_t nbr, const int32_t *__restrict__ bptr,
    const int32_t *__restrict__ bcol, const T *__restrict__ bval, const T *__restrict__ B, int64_t ldb,
    float *__restrict__ C, int64_t ldc, float alpha, float beta, int32_t *__restrict__ err) {
  __shared__ SpmmStage<NT> ring[kWarpsPerCta][kStages];
  __shared__ uint64_t bars[kWarpsPerCta][kStages];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  SpmmStage<NT> *st = ring[w];
  uint64_t *bar = bars[w];
  if (lane == 0) {
    for (int i = 0; i < kStages; ++i) mbar_init(&bar[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const int nchunks = N / (8 * NT);
  const int64_t items = (int64_t)nbr * nchunks;
  const int64_t gw = (int64_t)blockIdx.x * kWarpsPerCta + w;
  const int64_t nw = (int64_t)gridDim.x * kWarpsPerCta;
  unsigned uses[kStages];
#pragma unroll
  for (int i = 0; i < kStages; ++i) uses[i] = 0;
  const int g = lane >> 2, t4 = lane & 3;
  for (int64_t item = gw; item < items; item += nw) {
    const int32_t br = (int32_t)(item / nchunks);
    const int32_t n0 = (int32_t)(item % nchunks) * 8 * NT;
    const int32_t k0 = bptr[br], k1 = bptr[br + 1];
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    // producer (lane 0): stage tile k into slot k % kStages
    auto issue = [&](int32_t k) {
      const int slot = (k - k0) % kStages;
      SpmmStage<NT> &S = st[slot];
      const int32_t bc = bcol[k];
      int rows_in = K - bc * kTS;
      rows_in = rows_in > kTS ? kTS : rows_in;
      const unsigned bytes = kTS * kTS * 2 + (unsigned)rows_in * (8 * NT * 2);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&bar[slot], bytes);
      bulk_g2s(S.a, bval + (int64_t)k * kTS * kTS, kTS * kTS * 2, &bar[slot]);
      for (int rr = 0; rr < rows_in; ++rr)
        bulk_g2s(S.b + rr * SpmmStage<NT>::kBStride, B + ((int64_t)bc * kTS + rr) * ldb + n0, 8 * NT * 2,
                 &bar[slot]);
    };
    // rows of B beyond K are never copied: zero them (generic proxy) and
    // order those writes before the slot's next asynchronous copies
    auto zero_tail = [&](SpmmStage<NT> &S, int32_t k) {
      const int32_t bc = bcol[k];
      const int64_t rows_in = (int64_t)K - (int64_t)bc * kTS;
      if (rows_in < kTS) {
        constexpr int kWords = SpmmStage<NT>::kBStride / 4;
        uint32_t *tail = reinterpret_cast<uint32_t *>(S.b + rows_in * SpmmStage<NT>::kBStride);
        for (int i = lane; i < (kTS - (int)rows_in) * kWords; i += 32) tail[i] = 0u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
      }
    };
    const int32_t nk = k1 - k0;
    for (int32_t k = k0; k < k0 + (nk < kStages ? nk : kStages); ++k) {
      zero_tail(st[(k - k0) % kStages], k);
      if (lane == 0) issue(k);
    }
    bool ok = true;
    for (int32_t k = k0; k < k1; ++k) {
      const int slot = (k - k0) % kStages;
      if (!mbar_wait(&bar[slot], uses[slot] & 1u)) {
        ok = false;
        break;
      }
      uses[slot]++;
      SpmmStage<NT> &S = st[slot];
      uint32_t a[4];
      ldm_x4(a, S.a + tile_pos(lane & 15, (lane >> 4) * 8) * 2);
#pragma unroll
      for (int j = 0; j < NT; j += 2) {
        uint32_t b[4];
        ldm_x4_trans(b, S.b + (lane & 15) * SpmmStage<NT>::kBStride + (8 * j + 8 * (lane >> 4)) * 2);
        mma16816<T>(acc[j], a, b[0], b[1]);
        mma16816<T>(acc[j + 1], a, b[2], b[3]);
      }
      __syncwarp();  // every lane has read the slot before it is refilled
      const int32_t kn = k + kStages;
      if (kn < k1) {
        zero_tail(S, kn);
        if (lane == 0) issue(kn);
      }
    }
    if (!ok) {
      if (lane == 0) atomicExch(err, 1);
      // let this warp's own copies in flight land (bounded), then stop
      for (int i = 0; i < kStages; ++i) (void)mbar_wait(&bar[i], uses[i] & 1u);
      return;
    }
    // epilogue: C rows br*16 + g and + 8, columns n0 + 8j + 2*t4
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int32_t col = n0 + 8 * j + 2 * t4;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t row = (int64_t)br * kTS + g + 8 * h;
        if (row < M) {
          float *cp = C + row * ldc + col;
          float o0 = alpha * acc[j][2 * h], o1 = alpha * acc[j][2 * h + 1];
          if (beta != 0.f) {
            o0 += beta * cp[0];
            o1 += beta * cp[1];
          }
          cp[0] = o0;
          cp[1] = o1;
        }
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Block SpMM on the 5th-generation tensor cores (tcgen05), for N % 128 == 0.
//
// Transposed product: for a 16-row block br and a 128-column slab n0 of C,
//   D (128 x 16, FP32, in tensor memory) = sum over the block-row's tiles of
//   Bslab^T (128 x 16: rows bc*16.. of B, columns n0..n0+127) * Atile^T.
// D's row m is C column n0+m, its column j is C row br*16+j.  One
// tcgen05.mma (kind::f16, M = 128, N = 16, K = 16) per tile:
//   * A operand = the B slab, MN-major, loaded by TMA (two 64-column boxes,
//     128-byte swizzle) into a 4 KB stage aligned to 1 KB;
//   * B operand = the stored tile (512 B, no swizzle, K-major core matrices,
//     see tile_pos) copied with cp.async.bulk.
// Thread 0 runs a kTcStages-deep pipeline (4 stages keep ~11 CTAs per SM): wait for a stage's bytes, issue
// the MMA, commit it to the stage's "empty" barrier, refill the stage when
// that MMA has read it.  A final commit signals the epilogue: every warp
// reads its 32 TMEM lanes (tcgen05.ld 32x32b, 16 columns) and writes 16 C
// rows for its 32 columns.  Waits are bounded; on a timeout the kernel
// records an error, waits (bounded) for its own copies, frees its TMEM and
// returns.  Rows of B past K come back as zeros from TMA.
constexpr int kTcStages = 4;
constexpr int kTcSlab = 128;                       // UMMA M = C columns per CTA
constexpr int kTcBBytes = kTcSlab * kTS * 2;       // 4096
constexpr int kTcABytes = kTS * kTS * 2;           // 512
constexpr int kTcThreads = 128;
constexpr int kTcTmemCols = 32;                    // >= N = 16, power of two
constexpr int kTcSmem = 1024 + kTcStages * (kTcBBytes + kTcABytes) + 128;

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // sm100 descriptor version
  d |= (uint64_t)(layout & 7u) << 61;
  return d;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int32_t c0, int32_t c1,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// W (64 or 128) = C columns per CTA.  With W = 64 only the first 64-column
// box of each stage is loaded and the MMA's rows 64..127 (whatever the stage
// held) are never read back; this halves the B slab (B rows x W) that the
// CTAs of one slab pass keep in L2.  Columns at or past N are zero-filled by
// TMA and not stored.
template <typename T>
__global__ void __launch_bounds__(kTcThreads) spmm_tc_kernel(const __grid_constant__ CUtensorMap tmB, int32_t M,
                                                             int32_t N, int32_t W, int32_t nbr,
                                                             const int32_t *__restrict__ bptr,
                                                             const int32_t *__restrict__ bcol,
                                                             const T *__restrict__ tiles, float *__restrict__ C,
                                                             int64_t ldc, float alpha, float beta,
                                                             int32_t *__restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + ((1024u - (raw & 1023u)) & 1023u);  // 1 KB aligned for the swizzle atoms
  unsigned char *bslab = sm;
  unsigned char *atile = sm + kTcStages * kTcBBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(atile + kTcStages * kTcABytes);
  uint64_t *empty = full + kTcStages;
  uint64_t *done = empty + kTcStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t br = blockIdx.x;
  const int32_t n0 = blockIdx.y * W;
  const bool two_boxes = W > 64;
  const int32_t k0 = bptr[br], nk = bptr[br + 1] - k0;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kTcStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)kTcTmemCols)
                 : "memory");
    // this CTA allocates only once: let the other CTAs on the SM allocate
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  int ok = 1;
  if (threadIdx.x == 0 && nk > 0) {
    constexpr uint32_t fmt = std::is_same<T, __nv_bfloat16>::value ? 1u : 0u;
    // kind::f16 instruction descriptor: D FP32, A and B in `fmt`, A MN-major,
    // B K-major, N = 16, M = 128
    constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | (1u << 15) | ((16u >> 3) << 17) |
                               ((uint32_t)(kTcSlab >> 4) << 24);
    int issued = 0, waited = 0;
    auto load = [&](int i) {
      const int st = i % kTcStages;
      const int32_t bc = bcol[k0 + i];
      mbar_expect_tx(&full[st], (two_boxes ? kTcBBytes : kTcBBytes / 2) + kTcABytes);
      tma_load_2d(bslab + st * kTcBBytes, &tmB, n0, bc * kTS, &full[st]);
      if (two_boxes) tma_load_2d(bslab + st * kTcBBytes + kTcBBytes / 2, &tmB, n0 + 64, bc * kTS, &full[st]);
      bulk_g2s(atile + st * kTcABytes, tiles + (int64_t)(k0 + i) * kTS * kTS, kTcABytes, &full[st]);
      ++issued;
    };
    for (int i = 0; i < nk && i < kTcStages; ++i) load(i);
    for (int i = 0; i < nk; ++i) {
      const int st = i % kTcStages;
      const unsigned ph = (unsigned)(i / kTcStages) & 1u;
      if (!mbar_wait(&full[st], ph)) {
        ok = 0;
        break;
      }
      ++waited;
      // A: the B slab, 128-byte swizzle, 64-column halves 2 KB apart (LBO),
      // 8-row K groups 1 KB apart (SBO).  B: the tile, no swizzle, K halves
      // 128 B apart (LBO), 8-row groups 256 B apart (SBO).
      const uint64_t adesc = umma_smem_desc(smem_u32(bslab + st * kTcBBytes), 2048u, 1024u, 2u);
      const uint64_t bdesc = umma_smem_desc(smem_u32(atile + st * kTcABytes), 128u, 256u, 0u);
      umma_f16(tmem, adesc, bdesc, idesc, i > 0 ? 1u : 0u);
      umma_commit(&empty[st]);
      if (i + kTcStages < nk) {
        if (!mbar_wait(&empty[st], ph)) {  // this stage's MMA has read it
          ok = 0;
          break;
        }
        load(i + kTcStages);
      }
    }
    umma_commit(done);  // arrives when every MMA issued above has completed
    if (!ok) {
      // let the copies still in flight land before the CTA goes away
      for (int j = waited; j < issued; ++j) (void)mbar_wait(&full[j % kTcStages], (unsigned)(j / kTcStages) & 1u);
    }
  }
  __syncwarp();
  int good = ok;
  if (nk > 0) good = good && mbar_wait(done, 0u);
  const int all_good = __syncthreads_and(good);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  float v[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = 0.f;
  if (all_good && nk > 0) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
  }
  if (all_good) {
    const int64_t col = (int64_t)n0 + warp * 32 + lane;
    const bool mine = warp * 32 < W && col < N;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t row = (int64_t)br * kTS + j;
      if (mine && row < M) {
        float *cp = C + row * ldc + col;
        *cp = scale_out(alpha, v[j], beta, cp);
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcTmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Persistent, warp-specialised form of the tcgen05 block SpMM.  The CTAs of
// one launch stay resident and walk the work items w = blockIdx.x +
// j * gridDim.x (item = (16-row block br, slab of WT C columns), slab-major),
// so the set-up (barriers, TMEM allocation) is paid once per CTA instead of
// once per block row, and the tile stream runs on across block rows:
//   warp 0 (one lane): producer -- per tile, waits for its stage to be free,
//     then TMA-loads the B slab box(es) and bulk-copies the stored tile;
//   warp 1 (one lane): MMA issuer -- per tile one tcgen05.mma into the item's
//     accumulator (TMEM columns 16 * (j & 1): two accumulators, so block row
//     j + 1 accumulates while block row j is read out), commit frees the
//     stage; after an item's last tile a commit signals the epilogue;
//   warps 2-5: epilogue -- each reads its quarter of the TMEM lanes
//     (tcgen05.ld 32x32b.x16: 32 C columns x 16 C rows), hands the
//     accumulator back, and writes C.
// Every wait is bounded; a timeout sets the shared abort flag, which the
// other roles see at their next wait, and the error flag; the producer then
// waits (bounded) for the copies it issued before leaving.
//
// WT = 64 or 128 C columns per item, S stages of 128 x 16 B values (one or
// two 64-column TMA boxes) + one 512-byte tile.  With WT = 64 the MMA still
// has M = 128: its A rows 64..127 read the stage's upper 2 KB, which no copy
// writes (a stride of 2 KB, with those rows reading the next stage while TMA
// filled it, measured 1.4-2.5x slower at N = 128 / 256), and the matching D
// lanes are never read back.  HINT: L2 cache policies -- the B boxes are loaded evict-last (a
// slab pass re-reads each B block row once per tile that uses it), the tiles
// evict-first and C stored streaming, so that the one-use data does not push
// B out of L2.
constexpr int kTcpThreads = 192;

template <int WT, int S>
struct TcpCfg {
  static constexpr int kBBytes = kTcSlab * kTS * 2;   // stage stride: the MMA's 128 A rows
  static constexpr int kLoadBytes = WT * kTS * 2;     // what the boxes bring
  static constexpr int kSmem = 1024 + S * (kBBytes + kTcABytes) + 256;
  static_assert(WT == 64 || WT == 128, "slab width");
};

__device__ __forceinline__ bool tcp_wait(uint64_t *bar, unsigned parity, volatile int *abort_flag) {
  for (long long i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 1023) == 1023 && *abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void tma_load_2d_hint(void *dst, const CUtensorMap *map, int32_t c0, int32_t c1,
                                                 uint64_t *bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, "
      "%3}], [%4], %5;" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
      "%4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// The items w = blockIdx.x + j * gridDim.x of an n x nslab item grid as
// (r, s) = (w % n, w / n), stepped without a division per item.
struct ItemWalk {
  int32_t r, s, dr, ds, n;
  __device__ __forceinline__ explicit ItemWalk(int32_t n_) : n(n_) {
    r = (int32_t)(blockIdx.x % (unsigned)n_);
    s = (int32_t)(blockIdx.x / (unsigned)n_);
    dr = (int32_t)(gridDim.x % (unsigned)n_);
    ds = (int32_t)(gridDim.x / (unsigned)n_);
  }
  __device__ __forceinline__ void next() {
    r += dr;
    s += ds;
    if (r >= n) {
      r -= n;
      ++s;
    }
  }
};

template <typename T, int WT, int S, bool HINT>
__global__ void __launch_bounds__(kTcpThreads) spmm_tcp_kernel(const __grid_constant__ CUtensorMap tmB, int32_t M,
                                                               int32_t N, int32_t col0, int32_t nslab,
                                                               int32_t nbr, const int32_t *__restrict__ bptr,
                                                               const int32_t *__restrict__ bcol,
                                                               const T *__restrict__ tiles, float *__restrict__ C,
                                                               int64_t ldc, float alpha, float beta,
                                                               int32_t *__restrict__ err) {
  using Cfg = TcpCfg<WT, S>;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  unsigned char *bslab = sm;
  unsigned char *atile = sm + S * Cfg::kBBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(atile + S * kTcABytes);
  uint64_t *empty = full + S;
  uint64_t *done = empty + S;           // [2]
  uint64_t *accfree = done + 2;         // [2]
  uint64_t *drain = accfree + 2;        // the MMA issuer's last commit
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&done[i], 1);
      mbar_init(&accfree[i], 4);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer
    const uint64_t keep = HINT ? l2_evict_last_policy() : 0, stream = HINT ? l2_evict_first_policy() : 0;
    int64_t it = 0;
    bool ok = true;
    for (ItemWalk iw(nbr); iw.s < nslab && ok; iw.next()) {
      const int32_t br = iw.r;
      const int32_t n0 = col0 + iw.s * WT;
      const int32_t k0 = bptr[br], nk = bptr[br + 1] - k0;
      for (int32_t i = 0; i < nk; ++i, ++it) {
        const int st = (int)(it % S);
        if (it >= S && !tcp_wait(&empty[st], (unsigned)((it / S - 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        const int32_t bc = bcol[k0 + i];
        unsigned char *bs = bslab + st * Cfg::kBBytes;
        const T *tp = tiles + (int64_t)(k0 + i) * kTS * kTS;
        mbar_expect_tx(&full[st], Cfg::kLoadBytes + kTcABytes);
        if (HINT) {
          tma_load_2d_hint(bs, &tmB, n0, bc * kTS, &full[st], keep);
          if (WT > 64) tma_load_2d_hint(bs + 2048, &tmB, n0 + 64, bc * kTS, &full[st], keep);
          bulk_g2s_hint(atile + st * kTcABytes, tp, kTcABytes, &full[st], stream);
        } else {
          tma_load_2d(bs, &tmB, n0, bc * kTS, &full[st]);
          if (WT > 64) tma_load_2d(bs + 2048, &tmB, n0 + 64, bc * kTS, &full[st]);
          bulk_g2s(atile + st * kTcABytes, tp, kTcABytes, &full[st]);
        }
      }
    }
    if (!ok) {
      // the copies issued into the last S stages land before the CTA goes away
      for (int64_t j = it > S ? it - S : 0; j < it; ++j) (void)mbar_wait(&full[j % S], (unsigned)((j / S) & 1));
      atomicExch(err, 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    constexpr uint32_t fmt = std::is_same<T, __nv_bfloat16>::value ? 1u : 0u;
    // kind::f16 instruction descriptor: D FP32, A and B in `fmt`, A MN-major,
    // B K-major, N = 16, M = 128
    constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | (1u << 15) | ((16u >> 3) << 17) |
                               ((uint32_t)(kTcSlab >> 4) << 24);
    int64_t it = 0, j = 0;
    bool ok = true;
    for (ItemWalk iw(nbr); iw.s < nslab && ok; iw.next(), ++j) {
      const int32_t br = iw.r;
      const int32_t nk = bptr[br + 1] - bptr[br];
      const int buf = (int)(j & 1);
      if (j >= 2 && !tcp_wait(&accfree[buf], (unsigned)((j / 2 - 1) & 1), abort_flag)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int32_t i = 0; i < nk; ++i, ++it) {
        const int st = (int)(it % S);
        if (!tcp_wait(&full[st], (unsigned)((it / S) & 1), abort_flag)) {
          ok = false;
          break;
        }
        // A: the B slab, 128-byte swizzle, 64-column halves 2 KB apart (LBO),
        // 8-row K groups 1 KB apart (SBO).  B: the tile, no swizzle, K halves
        // 128 B apart (LBO), 8-row groups 256 B apart (SBO).
        const uint64_t adesc = umma_smem_desc(smem_u32(bslab + st * Cfg::kBBytes), 2048u, 1024u, 2u);
        const uint64_t bdesc = umma_smem_desc(smem_u32(atile + st * kTcABytes), 128u, 256u, 0u);
        umma_f16(tmem + 16u * (uint32_t)buf, adesc, bdesc, idesc, i > 0 ? 1u : 0u);
        umma_commit(&empty[st]);
      }
      umma_commit(&done[buf]);   // arrives when every MMA issued so far has completed
    }
    // no MMA may still be writing TMEM when the CTA frees it
    umma_commit(drain);
    if (!mbar_wait(drain, 0u)) ok = false;
    if (!ok) atomicExch(err, 1);
  } else if (warp >= 2) {
    // ---- epilogue: warp w reads TMEM lanes 32 * (w % 4) .. + 31
    const int q = warp & 3;
    int64_t j = 0;
    for (ItemWalk iw(nbr); iw.s < nslab; iw.next(), ++j) {
      const int32_t br = iw.r;
      const int32_t n0 = col0 + iw.s * WT;
      const int32_t nk = bptr[br + 1] - bptr[br];
      const int buf = (int)(j & 1);
      if (!tcp_wait(&done[buf], (unsigned)((j / 2) & 1), abort_flag)) {
        atomicExch(err, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = 0.f;
      if (nk > 0) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)(q * 32) << 16) + 16u * (uint32_t)buf));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r[c]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&accfree[buf]);
      const int64_t col = (int64_t)n0 + q * 32 + lane;
      if (q * 32 < WT && col < N) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int64_t row = (int64_t)br * kTS + r;
          if (row < M) {
            float *cp = C + row * ldc + col;
            const float o = scale_out(alpha, v[r], beta, cp);
            if (HINT)
              __stcs(cp, o);
            else
              *cp = o;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcTmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Gathered-tile tensor-core SpMM (bsp_gtile): for matrices whose nonzeros
// scatter over all columns (graph adjacency), 16x16 tiles of the matrix as
// given are almost empty.  Here every 16-row group's distinct columns are
// compacted: chunk c of a group holds 16 of them (chunk_cols) and the 16x16
// tile of the group's values in those columns (chunk_tiles, the K-major core
// layout of tile_pos).  The product of a chunk is D (C columns x 16 rows) +=
// Bg^T x tile^T, Bg = the 16 gathered B rows: the same tcgen05.mma as the
// block kernel, with the B rows gathered by the producer warp (cp.async, 16
// bytes per lane and copy, written in the 128-byte swizzled layout the TMA
// would produce) instead of one TMA box.  Structure as spmm_tcp_kernel:
// resident CTAs walk (piece, slab) items, a piece being a run of up to
// kGtPieceChunks chunks of one group; groups with several pieces write
// partial rows, summed in piece order by gtile_reduce_kernel.
constexpr int kGtPieceChunks = 64;
constexpr int kGtcSmem = TcpCfg<128, kTcStages>::kSmem;
constexpr bool kGtcPerSlab = true;

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kTcpThreads) spmm_gtc_kernel(
    int32_t M, int32_t N, int32_t W, int32_t col0, int32_t nslab, int32_t npieces,
    const int32_t *__restrict__ piece_ptr,
    const int32_t *__restrict__ piece_group, const int32_t *__restrict__ piece_slot,
    const int32_t *__restrict__ chunk_cols, const T *__restrict__ tiles, const T *__restrict__ B, int64_t ldb,
    float *__restrict__ C, int64_t ldc, float *__restrict__ part, float alpha, float beta,
    int32_t *__restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  unsigned char *bslab = sm;
  unsigned char *atile = sm + kTcStages * kTcBBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(atile + kTcStages * kTcABytes);
  uint64_t *empty = full + kTcStages;
  uint64_t *done = empty + kTcStages;   // [2]
  uint64_t *accfree = done + 2;         // [2]
  uint64_t *drain = accfree + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kTcStages; ++i) {
      mbar_init(&full[i], 33);   // 32 cp.async arrivals + the tile copy's expect_tx
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&done[i], 1);
      mbar_init(&accfree[i], 4);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---- producer warp: gathers 16 B rows per chunk, lane 0 copies the tile
    const int cpr = W / 8;   // 16-byte pieces per gathered row
    int64_t it = 0;
    bool ok = true;
    for (ItemWalk iw(npieces); iw.s < nslab && ok; iw.next()) {
      const int32_t p = iw.r;
      const int32_t n0 = col0 + iw.s * W;
      const int32_t c0 = piece_ptr[p], c1 = piece_ptr[p + 1];
      for (int32_t c = c0; c < c1; ++c, ++it) {
        const int st = (int)(it % kTcStages);
        int good = 1;
        if (lane == 0 && it >= kTcStages)
          good = tcp_wait(&empty[st], (unsigned)((it / kTcStages - 1) & 1), abort_flag) ? 1 : 0;
        good = __shfl_sync(0xffffffffu, good, 0);
        if (!good) {
          ok = false;
          break;
        }
        const int32_t col_l = lane < 16 ? chunk_cols[(int64_t)c * 16 + lane] : 0;
        unsigned char *dst0 = bslab + st * kTcBBytes;
        for (int q = lane; q < 16 * cpr; q += 32) {   // same trip count on every lane
          const int k = q / cpr, j = q % cpr;
          const int32_t brow = __shfl_sync(0xffffffffu, col_l, k);
          const int32_t cc = n0 + j * 8;
          const bool valid = cc < N;
          const T *src = valid ? B + (int64_t)brow * ldb + cc : B;
          unsigned char *dst = dst0 + (j >> 3) * 2048 + k * 128 + (((j & 7) ^ (k & 7)) << 4);
          cp_async16(dst, src, valid);
        }
        if (lane == 0) {
          mbar_expect_tx(&full[st], kTcABytes);
          bulk_g2s(atile + st * kTcABytes, tiles + (int64_t)c * kTS * kTS, kTcABytes, &full[st]);
        }
        cp_async_arrive_noinc(&full[st]);
      }
    }
    if (!ok) {
      if (lane == 0) {
        for (int64_t j = it > kTcStages ? it - kTcStages : 0; j < it; ++j)
          (void)mbar_wait(&full[j % kTcStages], (unsigned)((j / kTcStages) & 1));
        atomicExch(err, 1);
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    constexpr uint32_t fmt = std::is_same<T, __nv_bfloat16>::value ? 1u : 0u;
    constexpr uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | (1u << 15) | ((16u >> 3) << 17) |
                               ((uint32_t)(kTcSlab >> 4) << 24);
    int64_t it = 0, j = 0;
    bool ok = true;
    for (ItemWalk iw(npieces); iw.s < nslab && ok; iw.next(), ++j) {
      const int32_t p = iw.r;
      const int32_t nk = piece_ptr[p + 1] - piece_ptr[p];
      const int buf = (int)(j & 1);
      if (j >= 2 && !tcp_wait(&accfree[buf], (unsigned)((j / 2 - 1) & 1), abort_flag)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int32_t i = 0; i < nk; ++i, ++it) {
        const int st = (int)(it % kTcStages);
        if (!tcp_wait(&full[st], (unsigned)((it / kTcStages) & 1), abort_flag)) {
          ok = false;
          break;
        }
        // the gathered rows were written through the generic proxy (cp.async)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint64_t adesc = umma_smem_desc(smem_u32(bslab + st * kTcBBytes), 2048u, 1024u, 2u);
        const uint64_t bdesc = umma_smem_desc(smem_u32(atile + st * kTcABytes), 128u, 256u, 0u);
        umma_f16(tmem + 16u * (uint32_t)buf, adesc, bdesc, idesc, i > 0 ? 1u : 0u);
        umma_commit(&empty[st]);
      }
      umma_commit(&done[buf]);
    }
    umma_commit(drain);
    if (!mbar_wait(drain, 0u)) ok = false;
    if (!ok) atomicExch(err, 1);
  } else if (warp >= 2) {
    // ---- epilogue
    const int q = warp & 3;
    int64_t j = 0;
    for (ItemWalk iw(npieces); iw.s < nslab; iw.next(), ++j) {
      const int32_t p = iw.r;
      const int32_t n0 = col0 + iw.s * W;
      const int32_t nk = piece_ptr[p + 1] - piece_ptr[p];
      const int32_t g = piece_group[p], slot = piece_slot[p];
      const int buf = (int)(j & 1);
      if (!tcp_wait(&done[buf], (unsigned)((j / 2) & 1), abort_flag)) {
        atomicExch(err, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = 0.f;
      if (nk > 0) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(tmem + ((uint32_t)(q * 32) << 16) + 16u * (uint32_t)buf));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r[c]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&accfree[buf]);
      const int64_t col = (int64_t)n0 + q * 32 + lane;
      if (q * 32 < W && col < N) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int64_t row = (int64_t)g * kTS + r;
          if (row >= M) continue;
          if (slot >= 0) {
            part[((int64_t)slot * kTS + r) * N + col] = v[r];
          } else {
            float *cp = C + row * ldc + col;
            *cp = scale_out(alpha, v[r], beta, cp);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcTmemCols)
                 : "memory");
}

// C rows of the groups split into several pieces: alpha * (sum of the
// pieces' partial rows, in piece order) + beta * C.  Thread per (row, column).
__global__ void gtile_reduce_kernel(int32_t nsplit, const int32_t *__restrict__ split_groups,
                                    const int32_t *__restrict__ group_piece, const int32_t *__restrict__ piece_slot,
                                    int32_t M, int32_t N, const float *__restrict__ part, float *__restrict__ C,
                                    int64_t ldc, float alpha, float beta) {
  const int64_t total = (int64_t)nsplit * kTS * N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t col = (int32_t)(i % N);
    const int32_t r = (int32_t)((i / N) % kTS);
    const int32_t g = split_groups[i / ((int64_t)N * kTS)];
    const int64_t row = (int64_t)g * kTS + r;
    if (row >= M) continue;
    float acc = 0.f;
    for (int32_t p = group_piece[g]; p < group_piece[g + 1]; ++p)
      acc += part[((int64_t)piece_slot[p] * kTS + r) * N + col];
    float *cp = C + row * ldc + col;
    *cp = scale_out(alpha, acc, beta, cp);
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// B (K rows x N columns, row stride ldb elements) as a 2-D tensor map with
// 64-column x 16-row boxes and 128-byte swizzle.
static bsp_status make_b_map(CUtensorMap *map, const void *B, int32_t K, int32_t N, int64_t ldb, bool bf16) {
  auto enc = tensor_map_encoder();
  if (!enc) BSP_FAIL(BSP_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)K};
  const cuuint64_t strides[1] = {(cuuint64_t)ldb * 2};
  const cuuint32_t box[2] = {64, (cuuint32_t)kTS};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                         const_cast<void *>(B), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) BSP_FAIL(BSP_ERR_INVALID, "cuTensorMapEncodeTiled rejected B (code " + std::to_string((int)r) + ")");
  return BSP_OK;
}

template <typename T>
__device__ __forceinline__ T tile_cvt(double v);
template <> __device__ __forceinline__ __half tile_cvt<__half>(double v) { return __double2half(v); }
template <> __device__ __forceinline__ __nv_bfloat16 tile_cvt<__nv_bfloat16>(double v) {
  return __float2bfloat16_rn((float)v);
}

// Row-major FP64 tiles -> stored low-precision tiles.
template <typename T>
__global__ void tiles_to_lp_kernel(int64_t n, const double *__restrict__ v, T *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(i & 255);
    out[(i & ~(int64_t)255) + tile_pos(e >> 4, e & 15)] = tile_cvt<T>(v[i]);
  }
}

template <typename T, int CPL>
static bsp_status launch_spmm_csr(int32_t rows, int32_t N, const int32_t *rp, const int32_t *ci, const void *val,
                                  const void *B, int64_t ldb, float *C, int64_t ldc, float a, float b,
                                  cudaStream_t s) {
  int64_t blocks = ceil_div(rows, 8);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_csr_kernel<T, CPL><<<(unsigned)blocks, 256, 0, s>>>(rows, N, rp, ci, (const T *)val, (const T *)B, ldb, C,
                                                           ldc, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename T, int LPR>
static bsp_status launch_grouped(int32_t rows, int32_t N, const int32_t *rp, const int32_t *ci, const void *val,
                                 const void *B, int64_t ldb, float *C, int64_t ldc, float a, float b,
                                 cudaStream_t s) {
  int64_t blocks = ceil_div(rows, 8);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_grouped_kernel<T, LPR><<<(unsigned)blocks, 256, 0, s>>>(rows, N, rp, ci, (const T *)val, (const T *)B, ldb,
                                                               C, ldc, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename T>
static bsp_status spmm_csr_typed(int32_t rows, int32_t N, const int32_t *rp, const int32_t *ci, const void *val,
                                 const void *B, int64_t ldb, float *C, int64_t ldc, float a, float b,
                                 cudaStream_t s) {
  switch (grouped_lpr<T>(N, B, ldb)) {
    case 32: return launch_grouped<T, 32>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    case 16: return launch_grouped<T, 16>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    case 8: return launch_grouped<T, 8>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    case 4: return launch_grouped<T, 4>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    case 2: return launch_grouped<T, 2>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    case 1: return launch_grouped<T, 1>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    default: break;
  }
  // widest per-lane vector that divides N/32 and keeps B loads aligned
  const size_t es = sizeof(T);
  const bool al16 = ((uintptr_t)B % 16 == 0) && ((ldb * es) % 16 == 0);
  const bool al8 = ((uintptr_t)B % 8 == 0) && ((ldb * es) % 8 == 0);
  if (es == 2) {
    if (N % 256 == 0 && al16) return launch_spmm_csr<T, 8>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    if (N % 128 == 0 && al8) return launch_spmm_csr<T, 4>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    if (N % 64 == 0 && ((uintptr_t)B % 4 == 0) && ((ldb * es) % 4 == 0))
      return launch_spmm_csr<T, 2>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
    return launch_spmm_csr<T, 1>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
  }
  if (N % 128 == 0 && al16) return launch_spmm_csr<T, 4>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
  if (N % 64 == 0 && al8) return launch_spmm_csr<T, 2>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
  return launch_spmm_csr<T, 1>(rows, N, rp, ci, val, B, ldb, C, ldc, a, b, s);
}

// Longest row (atomicMax of the row lengths).
__global__ void spmm_max_row_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, int32_t *__restrict__ out) {
  int32_t m = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    m = max(m, rowPtr[r + 1] - rowPtr[r]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// A row this long keeps one warp busy far past the rest of the launch: the
// plan-free call routes such matrices through a temporary row-split plan.
constexpr int32_t kSpmmLongRow = 8192;
constexpr int32_t kSpmmTempChunk = 256;

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_spmm_csr(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                   const int32_t *colIdx, const void *values, bsp_dtype dtype, const void *B,
                                   int32_t N, int64_t ldb, float *C, int64_t ldc, float alpha, float beta,
                                   bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0 && N >= 0, "negative size");
  if (rows == 0 || N == 0) return BSP_OK;
  BSP_CHECK_ARG(rowPtr && C && (nnz == 0 || (colIdx && values && B)), "null pointer");
  BSP_CHECK_ARG(ldb >= N && ldc >= N, "leading dimension smaller than N");
  cudaStream_t s = as_stream(stream);
  BSP_CHECK_ARG(dtype == BSP_F16 || dtype == BSP_BF16 || dtype == BSP_F32, "SpMM takes F16, BF16 or F32 values");
  // Rows far longer than the mean (power-law graphs) would serialize on one
  // warp: look up the longest row (skipped while the stream is captured,
  // since it reads a value back) and split such rows with a temporary plan.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BSP_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap == cudaStreamCaptureStatusNone && nnz > kSpmmLongRow) {
    int32_t *d_max = nullptr, h_max = 0;
    BSP_TRY(dalloc(&d_max, 1, s));
    BSP_CUDA(cudaMemsetAsync(d_max, 0, sizeof(int32_t), s));
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(rows, 256), (int64_t)sm_count() * 8));
    spmm_max_row_kernel<<<g, 256, 0, s>>>(rows, rowPtr, d_max);
    const bsp_status st = read_i32(d_max, &h_max, s);
    dfree(d_max, s);
    BSP_TRY(st);
    if (h_max > kSpmmLongRow && (int64_t)h_max > 64 * ((int64_t)nnz / rows + 1)) {
      bsp_spmm_plan plan{};
      BSP_TRY(bsp_spmm_plan_create(rows, nnz, rowPtr, kSpmmTempChunk, &plan, stream));
      const size_t ws = bsp_spmm_plan_workspace(&plan, N);
      void *work = nullptr;
      bsp_status r2 = BSP_OK;
      if (ws > 0 && cudaMallocAsync(&work, ws, s) != cudaSuccess) {
        set_error("bsp_spmm_csr: allocating the row-split workspace failed");
        r2 = BSP_ERR_ALLOC;
      }
      if (r2 == BSP_OK)
        r2 = bsp_spmm_csr_planned(&plan, cols, nnz, rowPtr, colIdx, values, dtype, B, N, ldb, C, ldc, alpha, beta,
                                  work, ws, stream);
      if (work) cudaFreeAsync(work, s);
      bsp_spmm_plan_free(&plan);
      return r2;
    }
  }
  switch (dtype) {
    case BSP_F16:
      return spmm_csr_typed<__half>(rows, N, rowPtr, colIdx, values, B, ldb, C, ldc, alpha, beta, s);
    case BSP_BF16:
      return spmm_csr_typed<__nv_bfloat16>(rows, N, rowPtr, colIdx, values, B, ldb, C, ldc, alpha, beta, s);
    case BSP_F32:
      return spmm_csr_typed<float>(rows, N, rowPtr, colIdx, values, B, ldb, C, ldc, alpha, beta, s);
    default:
      BSP_FAIL(BSP_ERR_UNSUPPORTED, "SpMM takes F16, BF16 or F32 values");
  }
}

extern "C" bsp_status bsp_smat_create(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                      const int32_t *colIdx, const double *values, bsp_dtype dtype, bsp_smat *out,
                                      bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out, "null output");
  BSP_CHECK_ARG(dtype == BSP_F16 || dtype == BSP_BF16, "block SpMM takes F16 or BF16");
  cudaStream_t s = as_stream(stream);
  bsp_smat m{};
  m.rows = rows;
  m.cols = cols;
  m.nnz = nnz;
  m.dtype = dtype;
  BSP_TRY(bsp_csr2bcsr(rows, cols, nnz, rowPtr, colIdx, values, kTS, kTS, 0, &m.tiles, stream));
  const int64_t ne = (int64_t)m.tiles.nonzeroBlocks * kTS * kTS;
  BSP_TRY(dalloc(reinterpret_cast<uint16_t **>(&m.tile_val), (size_t)(ne > 0 ? ne : 1), s));
  BSP_TRY(dalloc(&m.err, 1, s));
  BSP_CUDA(cudaMemsetAsync(m.err, 0, sizeof(int32_t), s));
  if (ne > 0) {
    int64_t g = ceil_div(ne, 256);
    if (g > (int64_t)sm_count() * 32) g = (int64_t)sm_count() * 32;
    if (dtype == BSP_F16)
      tiles_to_lp_kernel<__half><<<(unsigned)g, 256, 0, s>>>(ne, m.tiles.values, (__half *)m.tile_val);
    else
      tiles_to_lp_kernel<__nv_bfloat16><<<(unsigned)g, 256, 0, s>>>(ne, m.tiles.values,
                                                                    (__nv_bfloat16 *)m.tile_val);
    BSP_LAUNCH_CHECK();
  }
  // the FP64 tile values are not needed by the SpMM
  dfree(m.tiles.values, s);
  m.fill = m.tiles.nonzeroBlocks > 0 ? (double)nnz / ((double)m.tiles.nonzeroBlocks * kTS * kTS) : 0.0;
  BSP_CUDA(cudaStreamSynchronize(s));
  *out = m;
  return BSP_OK;
}

extern "C" bsp_status bsp_smat_free(bsp_smat *m) {
  clear_error();
  if (!m) return BSP_OK;
  cudaStream_t s = 0;
  if (m->tile_val) cudaFreeAsync(m->tile_val, s);
  m->tile_val = nullptr;
  dfree(m->err, s);
  BSP_TRY(bsp_bcsr_free(&m->tiles));
  return BSP_OK;
}

// Slab width of the one-CTA-per-block-row tcgen05 kernel when none is given:
// 128 columns per CTA for N >= 128, else 64.  Keeping a slab of B within L2
// by taking 64 columns at N >= 128 measured slower (N = 128: 431 vs 233 us):
// twice the CTAs, each paying its set-up.
static int tc_slab_width(int32_t N, int32_t cols) {
  (void)cols;
  return N >= 128 ? 128 : 64;
}

// Resident CTAs per SM for the persistent kernel: at most 8 (40 registers x
// 192 threads; TMEM 8 x 32 of 512 columns), fewer when the stages' shared
// memory (plus 1 KB the system keeps per CTA) does not fit 228 KB.  The
// occupancy API's answer here left one CTA per SM (148 CTAs, 9.4% of warps
// active).
static int tcp_blocks_per_sm(int smem) {
  const int by_smem = (228 * 1024) / (smem + 1024);
  return std::max(1, std::min(8, by_smem));
}

// Stages per slab width and whether the L2 policies are used.
constexpr int kTcpStages64 = 4;
constexpr int kTcpStages128 = 4;
constexpr bool kTcpHint = true;

template <typename T, int WT, int S>
static void tcp_launch(const CUtensorMap &map, const bsp_smat *m, int32_t N, float *C, int64_t ldc, float alpha,
                       float beta, cudaStream_t s) {
  using Cfg = TcpCfg<WT, S>;
  const int64_t total = (int64_t)m->tiles.rowRegions;
  const int per_sm = tcp_blocks_per_sm(Cfg::kSmem);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(total, (int64_t)sm_count() * per_sm));
  for (int32_t c0 = 0; c0 < N; c0 += WT)
    spmm_tcp_kernel<T, WT, S, kTcpHint><<<grid, kTcpThreads, Cfg::kSmem, s>>>(
        map, m->rows, N, c0, 1, m->tiles.rowRegions, m->tiles.bcsrRowPtr, m->tiles.bcsrcolIdx,
        (const T *)m->tile_val, C, ldc, alpha, beta, m->err);
}

// Persistent form: one wave of resident CTAs walking all block rows, one
// launch per slab of WT C columns.  A single launch over all slabs (items
// slab-major) let CTAs drift into the next slab while others finished the
// last, so two slabs of B competed for L2 (dense tiles, N = 256: 310 us with
// the item walk dividing per item, 329 us without; 64-column slabs 500 ->
// 1140 us); launches per slab keep one slab's B in flight at a time.
static bsp_status smat_spmm_tcp(const bsp_smat *m, const void *B, int32_t N, int64_t ldb, float *C, int64_t ldc,
                                float alpha, float beta, int32_t W, cudaStream_t s) {
  CUtensorMap map;
  BSP_TRY(make_b_map(&map, B, m->cols, N, ldb, m->dtype == BSP_BF16));
  const bool bf = m->dtype == BSP_BF16;
  if (W == 128) {
    if (bf)
      tcp_launch<__nv_bfloat16, 128, kTcpStages128>(map, m, N, C, ldc, alpha, beta, s);
    else
      tcp_launch<__half, 128, kTcpStages128>(map, m, N, C, ldc, alpha, beta, s);
  } else {
    if (bf)
      tcp_launch<__nv_bfloat16, 64, kTcpStages64>(map, m, N, C, ldc, alpha, beta, s);
    else
      tcp_launch<__half, 64, kTcpStages64>(map, m, N, C, ldc, alpha, beta, s);
  }
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

static bsp_status smat_spmm_tc(const bsp_smat *m, const void *B, int32_t N, int64_t ldb, float *C, int64_t ldc,
                               float alpha, float beta, int32_t W, cudaStream_t s) {
  CUtensorMap map;
  BSP_TRY(make_b_map(&map, B, m->cols, N, ldb, m->dtype == BSP_BF16));
  if (W == 0) W = tc_slab_width(N, m->cols);
  const dim3 grid((unsigned)m->tiles.rowRegions, (unsigned)ceil_div(N, W));
  if (m->dtype == BSP_F16)
    spmm_tc_kernel<__half><<<grid, kTcThreads, kTcSmem, s>>>(map, m->rows, N, W, m->tiles.rowRegions,
                                                             m->tiles.bcsrRowPtr, m->tiles.bcsrcolIdx,
                                                             (const __half *)m->tile_val, C, ldc, alpha, beta,
                                                             m->err);
  else
    spmm_tc_kernel<__nv_bfloat16><<<grid, kTcThreads, kTcSmem, s>>>(
        map, m->rows, N, W, m->tiles.rowRegions, m->tiles.bcsrRowPtr, m->tiles.bcsrcolIdx,
        (const __nv_bfloat16 *)m->tile_val, C, ldc, alpha, beta, m->err);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

extern "C" bsp_status bsp_smat_spmm(const bsp_smat *m, const void *B, int32_t N, int64_t ldb, float *C,
                                    int64_t ldc, float alpha, float beta, bsp_stream_t stream) {
  return bsp_smat_spmm_path(m, B, N, ldb, C, ldc, alpha, beta, BSP_SMAT_AUTO, stream);
}

extern "C" bsp_status bsp_smat_spmm_path(const bsp_smat *m, const void *B, int32_t N, int64_t ldb, float *C,
                                         int64_t ldc, float alpha, float beta, int32_t path,
                                         bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && B && C, "null pointer");
  BSP_CHECK_ARG(N > 0 && N % 32 == 0, "N must be a positive multiple of 32");
  BSP_CHECK_ARG(ldb >= N && ldc >= N, "leading dimension smaller than N");
  // cp.async.bulk needs 16-byte aligned sources and sizes
  BSP_CHECK_ARG((uintptr_t)B % 16 == 0 && (ldb * 2) % 16 == 0, "B must be 16-byte aligned with ldb % 8 == 0");
  BSP_CHECK_ARG((uintptr_t)m->tile_val % 16 == 0, "tile values must be 16-byte aligned");
  BSP_CHECK_ARG(path >= BSP_SMAT_AUTO && path <= BSP_SMAT_TCGEN05_PERSISTENT_W64, "unknown path");
  if (m->tiles.rowRegions == 0) return BSP_OK;
  cudaStream_t s = as_stream(stream);
  if (path == BSP_SMAT_TCGEN05_PERSISTENT)
    return smat_spmm_tcp(m, B, N, ldb, C, ldc, alpha, beta, N >= 128 ? 128 : 64, s);
  if (path == BSP_SMAT_TCGEN05_PERSISTENT_W64) return smat_spmm_tcp(m, B, N, ldb, C, ldc, alpha, beta, 64, s);
  if (path == BSP_SMAT_TCGEN05_W64) return smat_spmm_tc(m, B, N, ldb, C, ldc, alpha, beta, 64, s);
  if (path == BSP_SMAT_TCGEN05_W128) return smat_spmm_tc(m, B, N, ldb, C, ldc, alpha, beta, 128, s);
  // default tensor-core path: the persistent kernel (dense 16x16 tiles, 8 per
  // block row, 524,288 rows: N = 32 / 64 / 128 / 256 in 114 / 116 / 163 / 328
  // us, against 215 / 220 / 233 / 461 us with a CTA per block row and
  // 156 / 195 / 370 / 739 us on mma.sync)
  if (path == BSP_SMAT_TCGEN05 || path == BSP_SMAT_AUTO)
    return smat_spmm_tcp(m, B, N, ldb, C, ldc, alpha, beta, N >= 128 ? 128 : 64, s);
  const int nt = (N % 64 == 0) ? 8 : 4;
  const int64_t items = (int64_t)m->tiles.rowRegions * (N / (8 * nt));
  int64_t blocks = ceil_div(items, kWarpsPerCta);
  const int64_t cap = (int64_t)sm_count() * 16;
  if (blocks > cap) blocks = cap;
  const int32_t M = m->rows, K = m->cols, nbr = m->tiles.rowRegions;
#define BSP_SMAT_LAUNCH(T, NT)                                                                                 \
  spmm_block_kernel<T, NT><<<(unsigned)blocks, kWarpsPerCta * 32, 0, s>>>(                                   \
      M, K, N, nbr, m->tiles.bcsrRowPtr, m->tiles.bcsrcolIdx, (const T *)m->tile_val, (const T *)B, ldb, C, ldc, \
      alpha, beta, m->err)
  if (m->dtype == BSP_F16) {
    if (nt == 8)
      BSP_SMAT_LAUNCH(__half, 8);
    else
      BSP_SMAT_LAUNCH(__half, 4);
  } else {
    if (nt == 8)
      BSP_SMAT_LAUNCH(__nv_bfloat16, 8);
    else
      BSP_SMAT_LAUNCH(__nv_bfloat16, 4);
  }
#undef BSP_SMAT_LAUNCH
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

extern "C" bsp_status bsp_smat_check(const bsp_smat *m, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m, "null pointer");
  int32_t e = 0;
  BSP_TRY(read_i32(m->err, &e, as_stream(stream)));
  if (e) BSP_FAIL(BSP_ERR_TIMEOUT, "a bounded copy wait of the block SpMM timed out");
  return BSP_OK;
}

// ---------------------------------------------------------------------------
// Row-split CSR SpMM for power-law rows: a plan cuts every row longer than
// `chunk` nonzeros into chunks; one warp per chunk.  Chunks of a split row
// write their partial rows to a scratch buffer and a second kernel sums them
// in chunk order (deterministic, no atomics).
namespace bsp {

__global__ void spmm_plan_count_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, int32_t chunk,
                                       int32_t *__restrict__ nch, int32_t *__restrict__ npart) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t len = rowPtr[r + 1] - rowPtr[r];
    const int32_t c = len > chunk ? (len + chunk - 1) / chunk : 1;
    nch[r] = c;
    npart[r] = c > 1 ? c : 0;
  }
}

__global__ void spmm_plan_fill_kernel(int32_t rows, const int32_t *__restrict__ chunk_ptr,
                                      int32_t *__restrict__ chunk_row) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    for (int32_t c = chunk_ptr[r]; c < chunk_ptr[r + 1]; ++c) chunk_row[c] = (int32_t)r;
}

template <typename T, int CPL>
__global__ void __launch_bounds__(256) spmm_chunk_kernel(int64_t nchunks, int32_t N, int32_t chunk,
                                                         const int32_t *__restrict__ chunk_row,
                                                         const int32_t *__restrict__ chunk_ptr,
                                                         const int32_t *__restrict__ part_ptr,
                                                         const int32_t *__restrict__ rowPtr,
                                                         const int32_t *__restrict__ colIdx,
                                                         const T *__restrict__ val, const T *__restrict__ B,
                                                         int64_t ldb, float *__restrict__ C, int64_t ldc,
                                                         float *__restrict__ part, float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nchunks; w += nwarps) {
    const int32_t r = chunk_row[w];
    const int32_t ci = (int32_t)(w - chunk_ptr[r]);
    const bool split = chunk_ptr[r + 1] - chunk_ptr[r] > 1;
    const int32_t s0 = rowPtr[r], e0 = rowPtr[r + 1];
    const int32_t s = split ? s0 + ci * chunk : s0;
    const int32_t e = split ? min(s + chunk, e0) : e0;
    for (int32_t c0 = 0; c0 < N; c0 += 32 * CPL) {
      const int32_t cl = c0 + lane * CPL;
      const bool own = cl < N;
      float acc[CPL];
#pragma unroll
      for (int k = 0; k < CPL; ++k) acc[k] = 0.f;
      for (int32_t j0 = s; j0 < e; j0 += 32) {
        const int32_t j = j0 + lane;
        const int32_t cj = j < e ? colIdx[j] : 0;
        const float vj = j < e ? sp_to_float<T>(val[j]) : 0.f;
        const int cnt = e - j0 < 32 ? e - j0 : 32;
        int t = 0;
        for (; t + 4 <= cnt; t += 4) {
          float b[4][CPL];
          float v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int32_t c = __shfl_sync(0xffffffffu, cj, t + u);
            v[u] = __shfl_sync(0xffffffffu, vj, t + u);
            if (own) load_cols<T, CPL>(B + (int64_t)c * ldb + cl, b[u]);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < CPL; ++k) acc[k] = fmaf(v[u], b[u][k], acc[k]);
        }
        for (; t < cnt; ++t) {
          const int32_t c = __shfl_sync(0xffffffffu, cj, t);
          const float v = __shfl_sync(0xffffffffu, vj, t);
          float b[CPL];
          if (own) {
            load_cols<T, CPL>(B + (int64_t)c * ldb + cl, b);
#pragma unroll
            for (int k = 0; k < CPL; ++k) acc[k] = fmaf(v, b[k], acc[k]);
          }
        }
      }
      if (own) {
        if (split) {
          float *pp = part + ((int64_t)part_ptr[r] + ci) * N + cl;
#pragma unroll
          for (int k = 0; k < CPL; ++k) pp[k] = acc[k];
        } else {
          float *cp = C + (int64_t)r * ldc + cl;
#pragma unroll
          for (int k = 0; k < CPL; ++k) {
            float o = alpha * acc[k];
            if (beta != 0.f) o += beta * cp[k];
            cp[k] = o;
          }
        }
      }
    }
  }
}

// Split-row sums in two stages, so a row of many chunks (a 337,738-entry
// row is 1,320 chunks of 256) is not one warp's serial sum.  Stage one: a
// warp per group of up to 32 consecutive chunks of a row, lanes over the
// columns, 4 sums in flight per lane (chunk k into sum k % 4, added in a fixed
// order at the end); a row of one group is finished here.  Stage two: a warp
// per row of several groups adds its group sums the same way.
__device__ __forceinline__ float sum4_strided(const float *__restrict__ p, int64_t stride, int32_t n) {
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
  int32_t k = 0;
  for (; k + 3 < n; k += 4) {
    a0 += p[(int64_t)k * stride];
    a1 += p[(int64_t)(k + 1) * stride];
    a2 += p[(int64_t)(k + 2) * stride];
    a3 += p[(int64_t)(k + 3) * stride];
  }
  if (k < n) a0 += p[(int64_t)k * stride];
  if (k + 1 < n) a1 += p[(int64_t)(k + 1) * stride];
  if (k + 2 < n) a2 += p[(int64_t)(k + 2) * stride];
  return (a0 + a1) + (a2 + a3);
}

__device__ __forceinline__ void store_c(float *cp, float acc, float alpha, float beta) {
  float o = alpha * acc;
  if (beta != 0.f) o += beta * *cp;
  *cp = o;
}

__global__ void spmm_split_group_kernel(int32_t ngroups, const int32_t *__restrict__ group_split,
                                        const int32_t *__restrict__ group_ptr,
                                        const int32_t *__restrict__ split_rows,
                                        const int32_t *__restrict__ chunk_ptr,
                                        const int32_t *__restrict__ part_ptr, int32_t N,
                                        const float *__restrict__ part, float *__restrict__ gpart,
                                        float *__restrict__ C, int64_t ldc, float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups; g += nwarps) {
    const int32_t i = group_split[g];
    const int32_t r = split_rows[i];
    const int32_t nc = chunk_ptr[r + 1] - chunk_ptr[r];
    const int32_t gi = (int32_t)g - group_ptr[i];
    const int32_t k0 = gi * 32, n = min(32, nc - k0);
    const bool single = group_ptr[i + 1] - group_ptr[i] == 1;
    const float *pp = part + ((int64_t)part_ptr[r] + k0) * N;
    for (int32_t c = lane; c < N; c += 32) {
      const float acc = sum4_strided(pp + c, N, n);
      if (single)
        store_c(C + (int64_t)r * ldc + c, acc, alpha, beta);
      else
        gpart[g * N + c] = acc;
    }
  }
}

__global__ void spmm_split_rows_kernel(int32_t nsplit, const int32_t *__restrict__ split_rows,
                                       const int32_t *__restrict__ group_ptr, int32_t N,
                                       const float *__restrict__ gpart, float *__restrict__ C, int64_t ldc,
                                       float alpha, float beta) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nsplit; i += nwarps) {
    const int32_t g0 = group_ptr[i], ng = group_ptr[i + 1] - g0;
    if (ng <= 1) continue;   // finished by the group kernel
    const int32_t r = split_rows[i];
    const float *gp = gpart + (int64_t)g0 * N;
    for (int32_t c = lane; c < N; c += 32) store_c(C + (int64_t)r * ldc + c, sum4_strided(gp + c, N, ng), alpha, beta);
  }
}

// Groups of the split rows: ng[i] = ceil(chunks / 32) (scanned into
// group_ptr), then group_split lists the split row of every group.
__global__ void spmm_group_count_kernel(int32_t nsplit, const int32_t *__restrict__ split_rows,
                                        const int32_t *__restrict__ chunk_ptr, int32_t *__restrict__ ng) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nsplit; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == nsplit) {
      ng[i] = 0;
    } else {
      const int32_t r = split_rows[i];
      ng[i] = (chunk_ptr[r + 1] - chunk_ptr[r] + 31) / 32;
    }
  }
}

__global__ void spmm_group_fill_kernel(int32_t nsplit, const int32_t *__restrict__ group_ptr,
                                       int32_t *__restrict__ group_split) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nsplit; i += (int64_t)gridDim.x * blockDim.x)
    for (int32_t g = group_ptr[i]; g < group_ptr[i + 1]; ++g) group_split[g] = (int32_t)i;
}

// Sums the split rows' partials (`ncol` columns of `part`) into C; gpart
// holds the group sums of rows of more than 32 chunks.
static bsp_status split_reduce(const bsp_spmm_plan *p, int32_t ncol, const float *part, float *gpart, float *C,
                               int64_t ldc, float a, float b, cudaStream_t s) {
  if (p->nsplit <= 0) return BSP_OK;
  const int64_t cap = (int64_t)sm_count() * 32;
  const int64_t bg = std::min<int64_t>(std::max<int64_t>(1, ceil_div(p->ngroups, 8)), cap);
  spmm_split_group_kernel<<<(unsigned)bg, 256, 0, s>>>(p->ngroups, p->group_split, p->group_ptr, p->split_rows,
                                                      p->chunk_ptr, p->part_ptr, ncol, part, gpart, C, ldc, a, b);
  BSP_LAUNCH_CHECK();
  if (p->ngroups > p->nsplit) {   // some row has more than one group
    const int64_t br = std::min<int64_t>(std::max<int64_t>(1, ceil_div(p->nsplit, 8)), cap);
    spmm_split_rows_kernel<<<(unsigned)br, 256, 0, s>>>(p->nsplit, p->split_rows, p->group_ptr, ncol, gpart, C, ldc, a,
                                                       b);
    BSP_LAUNCH_CHECK();
  }
  return BSP_OK;
}

__global__ void spmm_split_list_kernel(int32_t rows, const int32_t *__restrict__ chunk_ptr,
                                       const int32_t *__restrict__ split_pos, int32_t *__restrict__ split_rows) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    if (chunk_ptr[r + 1] - chunk_ptr[r] > 1) split_rows[split_pos[r]] = (int32_t)r;
}

__global__ void spmm_long_chunk_kernel(int32_t rows, const int32_t *__restrict__ chunk_ptr,
                                       const int32_t *__restrict__ part_ptr, int32_t *__restrict__ long_chunk) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c0 = chunk_ptr[r], nc = chunk_ptr[r + 1] - c0;
    if (nc > 1)
      for (int32_t c = 0; c < nc; ++c) long_chunk[part_ptr[r] + c] = c0 + c;
  }
}

// Sort keys for the short-row list: chunk - length for rows of at most
// `chunk` nonzeros (so a stable ascending sort puts the longest first),
// chunk + 1 for split rows (sorted past the end of the list).
__global__ void spmm_short_key_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, int32_t chunk,
                                      int32_t *__restrict__ key, int32_t *__restrict__ idx) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t len = rowPtr[r + 1] - rowPtr[r];
    key[r] = len <= chunk ? chunk - len : chunk + 1;
    idx[r] = (int32_t)r;
  }
}

// Nonzero ranges for the slab engine: (start, end) of each partial-row
// slot's chunk and of each listed short row.
__global__ void spmm_range_kernel(int64_t nparts, const int32_t *__restrict__ long_chunk,
                                  const int32_t *__restrict__ chunk_row, const int32_t *__restrict__ chunk_ptr,
                                  int32_t chunk, int32_t nshort, const int32_t *__restrict__ short_rows,
                                  const int32_t *__restrict__ rowPtr, int2 *__restrict__ long_se,
                                  int2 *__restrict__ short_se) {
  const int64_t n = nparts > nshort ? nparts : nshort;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < nparts) {
      const int32_t w = long_chunk[i];
      const int32_t r = chunk_row[w];
      const int32_t st = rowPtr[r] + (w - chunk_ptr[r]) * chunk;
      long_se[i] = make_int2(st, min(st + chunk, rowPtr[r + 1]));
    }
    if (i < nshort) {
      const int32_t r = short_rows[i];
      short_se[i] = make_int2(rowPtr[r], rowPtr[r + 1]);
    }
  }
}

__global__ void spmm_split_flag_kernel(int32_t rows, const int32_t *__restrict__ chunk_ptr,
                                       int32_t *__restrict__ flag) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= rows; r += (int64_t)gridDim.x * blockDim.x)
    flag[r] = r < rows && chunk_ptr[r + 1] - chunk_ptr[r] > 1;
}

}  // namespace bsp

extern "C" bsp_status bsp_spmm_plan_create(int32_t rows, int32_t nnz, const int32_t *rowPtr, int32_t chunk,
                                           bsp_spmm_plan *out, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out && rowPtr && rows >= 0 && nnz >= 0, "bad argument");
  BSP_CHECK_ARG(chunk >= 32, "chunk must be >= 32");
  cudaStream_t s = as_stream(stream);
  bsp_spmm_plan p{};
  p.rows = rows;
  p.chunk = chunk;
  int32_t *flag = nullptr;
  int64_t *tot = nullptr;
  BSP_TRY(dalloc(&p.chunk_ptr, (size_t)rows + 1, s));
  BSP_TRY(dalloc(&p.part_ptr, (size_t)rows + 1, s));
  BSP_TRY(dalloc(&tot, 1, s));
  BSP_CUDA(cudaMemsetAsync(p.chunk_ptr + rows, 0, sizeof(int32_t), s));
  BSP_CUDA(cudaMemsetAsync(p.part_ptr + rows, 0, sizeof(int32_t), s));
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(rows + 1, 256), (int64_t)sm_count() * 32));
  if (rows > 0) {
    spmm_plan_count_kernel<<<g, 256, 0, s>>>(rows, rowPtr, chunk, p.chunk_ptr, p.part_ptr);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(exclusive_scan_i32(p.chunk_ptr, p.chunk_ptr, (int64_t)rows + 1, tot, s));
  int64_t h = 0;
  BSP_TRY(read_i64(tot, &h, s));
  p.nchunks = h;
  BSP_TRY(exclusive_scan_i32(p.part_ptr, p.part_ptr, (int64_t)rows + 1, tot, s));
  BSP_TRY(read_i64(tot, &h, s));
  p.nparts = h;
  BSP_TRY(dalloc(&p.chunk_row, (size_t)(p.nchunks > 0 ? p.nchunks : 1), s));
  if (rows > 0) {
    spmm_plan_fill_kernel<<<g, 256, 0, s>>>(rows, p.chunk_ptr, p.chunk_row);
    BSP_LAUNCH_CHECK();
  }
  BSP_TRY(dalloc(&flag, (size_t)rows + 1, s));
  spmm_split_flag_kernel<<<g, 256, 0, s>>>(rows, p.chunk_ptr, flag);
  BSP_LAUNCH_CHECK();
  BSP_TRY(exclusive_scan_i32(flag, flag, (int64_t)rows + 1, tot, s));
  BSP_TRY(read_i64(tot, &h, s));
  p.nsplit = (int32_t)h;
  BSP_TRY(dalloc(&p.split_rows, (size_t)(p.nsplit > 0 ? p.nsplit : 1), s));
  if (rows > 0) {
    spmm_split_list_kernel<<<g, 256, 0, s>>>(rows, p.chunk_ptr, flag, p.split_rows);
    BSP_LAUNCH_CHECK();
  }
  // reduce groups of the split rows
  BSP_TRY(dalloc(&p.group_ptr, (size_t)p.nsplit + 1, s));
  if (p.nsplit > 0) {
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div((int64_t)p.nsplit + 1, 256),
                                                                         (int64_t)sm_count() * 32));
    spmm_group_count_kernel<<<gs, 256, 0, s>>>(p.nsplit, p.split_rows, p.chunk_ptr, p.group_ptr);
    BSP_LAUNCH_CHECK();
  } else {
    BSP_CUDA(cudaMemsetAsync(p.group_ptr, 0, sizeof(int32_t), s));
  }
  BSP_TRY(exclusive_scan_i32(p.group_ptr, p.group_ptr, (int64_t)p.nsplit + 1, tot, s));
  BSP_TRY(read_i64(tot, &h, s));
  p.ngroups = (int32_t)h;
  BSP_TRY(dalloc(&p.group_split, (size_t)(p.ngroups > 0 ? p.ngroups : 1), s));
  if (p.nsplit > 0) {
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(p.nsplit, 256), (int64_t)sm_count() * 32));
    spmm_group_fill_kernel<<<gs, 256, 0, s>>>(p.nsplit, p.group_ptr, p.group_split);
    BSP_LAUNCH_CHECK();
  }
  dfree(flag, s);
  dfree(tot, s);
  // slab engine: the long chunks in partial-slot order, the short rows by length
  p.nshort = rows - p.nsplit;
  BSP_TRY(dalloc(&p.long_chunk, (size_t)(p.nparts > 0 ? p.nparts : 1), s));
  BSP_TRY(dalloc(&p.short_rows, (size_t)(rows > 0 ? rows : 1), s));
  if (rows > 0) {
    spmm_long_chunk_kernel<<<g, 256, 0, s>>>(rows, p.chunk_ptr, p.part_ptr, p.long_chunk);
    BSP_LAUNCH_CHECK();
    int32_t *keys = nullptr;
    BSP_TRY(dalloc(&keys, (size_t)rows, s));
    spmm_short_key_kernel<<<g, 256, 0, s>>>(rows, rowPtr, chunk, keys, p.short_rows);
    BSP_LAUNCH_CHECK();
    const bsp_status st = radix_sort_pairs(keys, p.short_rows, rows, bits_for(chunk + 1), s);
    dfree(keys, s);
    BSP_TRY(st);
  }
  BSP_TRY(dalloc(&p.long_se, (size_t)2 * (p.nparts > 0 ? p.nparts : 1), s));
  BSP_TRY(dalloc(&p.short_se, (size_t)2 * (p.nshort > 0 ? p.nshort : 1), s));
  if (p.nparts > 0 || p.nshort > 0) {
    const int64_t n = std::max<int64_t>(p.nparts, p.nshort);
    const unsigned gr = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)sm_count() * 32));
    spmm_range_kernel<<<gr, 256, 0, s>>>(p.nparts, p.long_chunk, p.chunk_row, p.chunk_ptr, chunk, p.nshort,
                                         p.short_rows, rowPtr, reinterpret_cast<int2 *>(p.long_se),
                                         reinterpret_cast<int2 *>(p.short_se));
    BSP_LAUNCH_CHECK();
  }
  p.slab_l2_hints = 1;
  BSP_CUDA(cudaStreamSynchronize(s));
  *out = p;
  return BSP_OK;
}

extern "C" bsp_status bsp_spmm_plan_free(bsp_spmm_plan *p) {
  clear_error();
  if (!p) return BSP_OK;
  cudaStream_t s = 0;
  dfree(p->chunk_ptr, s);
  dfree(p->part_ptr, s);
  dfree(p->chunk_row, s);
  dfree(p->split_rows, s);
  dfree(p->short_rows, s);
  dfree(p->long_chunk, s);
  dfree(p->long_se, s);
  dfree(p->short_se, s);
  dfree(p->group_ptr, s);
  dfree(p->group_split, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

namespace bsp {
// Warp per chunk (see spmm_chunk_kernel) with the grouped engine.
template <typename T, int LPR>
__global__ void __launch_bounds__(256, LPR >= 8 ? 6 : 0) spmm_grouped_chunk_kernel(
    int64_t nchunks, int32_t N, int32_t chunk, const int32_t *__restrict__ chunk_row,
    const int32_t *__restrict__ chunk_ptr, const int32_t *__restrict__ part_ptr, const int32_t *__restrict__ rowPtr,
    const int32_t *__restrict__ colIdx, const T *__restrict__ val, const T *__restrict__ B, int64_t ldb,
    float *__restrict__ C, int64_t ldc, float *__restrict__ part, float alpha, float beta) {
  constexpr int VEC = SpmmVec<T>::VEC;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nchunks; w += nwarps) {
    const int32_t r = chunk_row[w];
    const int32_t ci = (int32_t)(w - chunk_ptr[r]);
    const bool split = chunk_ptr[r + 1] - chunk_ptr[r] > 1;
    const int32_t s0 = rowPtr[r], e0 = rowPtr[r + 1];
    const int32_t s = split ? s0 + ci * chunk : s0;
    const int32_t e = split ? min(s + chunk, e0) : e0;
    for (int32_t c0 = 0; c0 < N; c0 += LPR * VEC) {
      const int32_t cl = c0 + (lane % LPR) * VEC;
      float acc[VEC];
#pragma unroll
      for (int k = 0; k < VEC; ++k) acc[k] = 0.f;
      spmm_segment<T, LPR>(s, e, colIdx, val, B, ldb, cl, lane, acc);
      if (lane < LPR) {
        if (split) {
          float *pp = part + ((int64_t)part_ptr[r] + ci) * N + cl;
#pragma unroll
          for (int k = 0; k < VEC; ++k) pp[k] = acc[k];
        } else {
          float *cp = C + (int64_t)r * ldc + cl;
#pragma unroll
          for (int k = 0; k < VEC; ++k) {
            float o = alpha * acc[k];
            if (beta != 0.f) o += beta * cp[k];
            cp[k] = o;
          }
        }
      }
    }
  }
}

template <typename T, int LPR>
static bsp_status launch_grouped_chunked(const bsp_spmm_plan *p, int32_t N, const int32_t *rp, const int32_t *ci,
                                         const void *val, const void *B, int64_t ldb, float *C, int64_t ldc,
                                         float *part, float a, float b, cudaStream_t s) {
  int64_t blocks = ceil_div(p->nchunks, 8);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_grouped_chunk_kernel<T, LPR><<<(unsigned)blocks, 256, 0, s>>>(
      p->nchunks, N, p->chunk, p->chunk_row, p->chunk_ptr, p->part_ptr, rp, ci, (const T *)val, (const T *)B, ldb, C,
      ldc, part, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename T, int CPL>
static bsp_status launch_chunked(const bsp_spmm_plan *p, int32_t N, const int32_t *rp, const int32_t *ci,
                                 const void *val, const void *B, int64_t ldb, float *C, int64_t ldc, float *part,
                                 float a, float b, cudaStream_t s) {
  int64_t blocks = ceil_div(p->nchunks, 8);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_chunk_kernel<T, CPL><<<(unsigned)blocks, 256, 0, s>>>(p->nchunks, N, p->chunk, p->chunk_row, p->chunk_ptr,
                                                             p->part_ptr, rp, ci, (const T *)val, (const T *)B, ldb,
                                                             C, ldc, part, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename T>
static bsp_status chunked_typed(const bsp_spmm_plan *p, int32_t N, const int32_t *rp, const int32_t *ci,
                                const void *val, const void *B, int64_t ldb, float *C, int64_t ldc, float *part,
                                float a, float b, cudaStream_t s) {
#define BSP_GC(L) launch_grouped_chunked<T, L>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s)
  switch (grouped_lpr<T>(N, B, ldb)) {
    case 32: return BSP_GC(32);
    case 16: return BSP_GC(16);
    case 8: return BSP_GC(8);
    case 4: return BSP_GC(4);
    case 2: return BSP_GC(2);
    case 1: return BSP_GC(1);
    default: break;
  }
#undef BSP_GC
  const size_t es = sizeof(T);
  const bool al16 = ((uintptr_t)B % 16 == 0) && ((ldb * es) % 16 == 0);
  const bool al8 = ((uintptr_t)B % 8 == 0) && ((ldb * es) % 8 == 0);
  if (es == 2) {
    if (N % 256 == 0 && al16) return launch_chunked<T, 8>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s);
    if (N % 128 == 0 && al8) return launch_chunked<T, 4>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s);
    return launch_chunked<T, 1>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s);
  }
  if (N % 128 == 0 && al16) return launch_chunked<T, 4>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s);
  return launch_chunked<T, 1>(p, N, rp, ci, val, B, ldb, C, ldc, part, a, b, s);
}

// ---------------------------------------------------------------------------
// Slab engine.  One pass per slab of NS = LPR*VEC columns [col0, col0 + NS):
// B's slab (B rows x NS) is small enough to stay in L2 for the whole pass, so
// every gathered B row after the first touch is an L2 hit, at the price of
// reading A once per slab.  Warp tasks [0, nlong) are the long rows' chunks,
// a warp each (G groups of LPR lanes split the chunk's nonzeros, then a
// fixed shuffle tree), written to their partial-row slot; the remaining tasks
// take G consecutive rows of the length-sorted short-row list, one row per
// group of LPR lanes, so a warp has G rows' load chains in flight at once
// instead of one.  Every task reads its nonzero range from the plan in one
// load (no slot -> chunk -> row -> rowPtr walk).  A chunk's next 32 column
// indices and values are loaded before the current 32 gathers are consumed;
// a short row's group loads its next U entries the same way.  With `hints`
// (bsp_spmm_plan.slab_l2_hints) 1 or 2, A's entries are loaded and C is
// stored evict-first, so the streamed A and C do not push the slab out of L2
// during the pass; with 1 the B rows are also gathered evict-last.
__device__ __forceinline__ uint64_t l2_policy(bool on, bool keep) {
  uint64_t p;
  if (!on)
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  else if (keep)
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  else
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ int32_t ld_hint_s32(const int32_t *p, uint64_t pol) {
  int32_t r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
  return r;
}
template <typename T> __device__ __forceinline__ float ld_hint_val(const T *p, uint64_t pol);
template <> __device__ __forceinline__ float ld_hint_val<float>(const float *p, uint64_t pol) {
  float r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r) : "l"(p), "l"(pol));
  return r;
}
template <> __device__ __forceinline__ float ld_hint_val<__half>(const __half *p, uint64_t pol) {
  unsigned short r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(r) : "l"(p), "l"(pol));
  return __half2float(__ushort_as_half(r));
}
template <> __device__ __forceinline__ float ld_hint_val<__nv_bfloat16>(const __nv_bfloat16 *p, uint64_t pol) {
  unsigned short r;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(r) : "l"(p), "l"(pol));
  return __bfloat162float(__ushort_as_bfloat16(r));
}
__device__ __forceinline__ uint4 ld_hint_b16(const void *p, uint64_t pol) {
  uint4 r;
  asm("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(pol));
  return r;
}

// Gathers in flight per lane group: U for a short row, UL per warp step of a
// long chunk.  8 at 4 lanes per B row (graph 2^20, FP16, N = 32) took 78
// registers and 0.551 ms (UL alone 0.605 ms, UL capped at 64 registers
// 0.507 ms) against 0.470 ms with 4.
template <int LPR> struct SlabU {
  static constexpr int U = 4;
  static constexpr int UL = 4;
};

template <typename T, int LPR, int U, int UL>
__global__ void __launch_bounds__(256, LPR >= 8 && LPR <= 16 ? (std::is_same<T, __nv_bfloat16>::value ? 4 : 5) : 0)
    spmm_slab_kernel(
    int64_t nlong, const int2 *__restrict__ long_se, int32_t nshort, const int32_t *__restrict__ short_rows,
    const int2 *__restrict__ short_se, const int32_t *__restrict__ colIdx, const T *__restrict__ val,
    const T *__restrict__ B, int64_t ldb, int32_t col0, float *__restrict__ C, int64_t ldc,
    float *__restrict__ part, float alpha, float beta, int32_t hints) {
  constexpr int VEC = SpmmVec<T>::VEC;
  constexpr int NS = LPR * VEC;
  constexpr int G = 32 / LPR;
  const int lane = threadIdx.x & 31;
  const int li = lane % LPR;
  const int g = lane / LPR;
  const int32_t cl = col0 + li * VEC;
  const uint64_t pa = l2_policy(hints != 0, false), pb = l2_policy(hints == 1, true);
  const int64_t ntasks = nlong + (nshort + G - 1) / G;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t task = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < ntasks; task += nwarps) {
    float acc[VEC];
#pragma unroll
    for (int k = 0; k < VEC; ++k) acc[k] = 0.f;
    if (task < nlong) {   // warp-uniform
      // Batches of BQ = 32*Q nonzeros: Q = 1 while a warp step's G*U gathers
      // fit in 32 (LPR >= 4), else one step takes the whole batch, so narrow
      // B rows still keep G*U gathers in flight per warp.
      constexpr int GU = G * UL;
      constexpr int Q = GU > 32 ? GU / 32 : 1;
      constexpr int BQ = 32 * Q;
      const int2 se = long_se[task];
      const int32_t e = se.y;
      int32_t cj[Q];
      float vj[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int32_t j = se.x + q * 32 + lane;
        cj[q] = j < e ? ld_hint_s32(colIdx + j, pa) : 0;
        vj[q] = j < e ? ld_hint_val<T>(val + j, pa) : 0.f;
      }
      for (int32_t j0 = se.x; j0 < e; j0 += BQ) {   // warp-uniform bounds
        int32_t cn[Q];
        float vn[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int32_t jn = j0 + BQ + q * 32 + lane;
          cn[q] = jn < e ? ld_hint_s32(colIdx + jn, pa) : 0;
          vn[q] = jn < e ? ld_hint_val<T>(val + jn, pa) : 0.f;
        }
        const int cnt = e - j0 < BQ ? e - j0 : BQ;
        for (int t = 0; t < cnt; t += GU) {   // one trip when Q > 1
          uint4 raw[UL];
          float v[UL];
#pragma unroll
          for (int u = 0; u < UL; ++u) {
            const int src = t + u * G + g;
            const int q = Q > 1 ? (u * G) >> 5 : 0;   // t == 0 when Q > 1
            const int32_t c = __shfl_sync(0xffffffffu, cj[q], src & 31);
            const float vv = __shfl_sync(0xffffffffu, vj[q], src & 31);
            const bool ok = src < cnt;
            v[u] = ok ? vv : 0.f;
            raw[u] = ok ? ld_hint_b16(B + (int64_t)c * ldb + cl, pb) : make_uint4(0, 0, 0, 0);
          }
#pragma unroll
          for (int u = 0; u < UL; ++u) {
            float b[VEC];
            unpack16<T>(raw[u], b);
#pragma unroll
            for (int k = 0; k < VEC; ++k) acc[k] = fmaf(v[u], b[k], acc[k]);
          }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          cj[q] = cn[q];
          vj[q] = vn[q];
        }
      }
#pragma unroll
      for (int o = LPR; o < 32; o <<= 1)
#pragma unroll
        for (int k = 0; k < VEC; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
      if (lane < LPR) {
        float *pp = part + task * NS + li * VEC;
#pragma unroll
        for (int k = 0; k < VEC; ++k) pp[k] = acc[k];
      }
      continue;
    }
    const int64_t i = (task - nlong) * G + g;
    if (i >= nshort) continue;
    const int32_t r = short_rows[i];
    const int2 se = short_se[i];
    const int32_t s = se.x, e = se.y;
    int32_t cn[U];
    float vn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool ok = s + u < e;
      cn[u] = ok ? ld_hint_s32(colIdx + s + u, pa) : 0;
      vn[u] = ok ? ld_hint_val<T>(val + s + u, pa) : 0.f;
    }
    for (int32_t j = s; j < e; j += U) {
      uint4 raw[U];
      float v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        v[u] = vn[u];
        raw[u] = j + u < e ? ld_hint_b16(B + (int64_t)cn[u] * ldb + cl, pb) : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int32_t jj = j + U + u;
        const bool ok = jj < e;
        cn[u] = ok ? ld_hint_s32(colIdx + jj, pa) : 0;
        vn[u] = ok ? ld_hint_val<T>(val + jj, pa) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        float b[VEC];
        unpack16<T>(raw[u], b);
#pragma unroll
        for (int k = 0; k < VEC; ++k) acc[k] = fmaf(v[u], b[k], acc[k]);
      }
    }
    float *cp = C + (int64_t)r * ldc + cl;
    if (beta != 0.f) {
#pragma unroll
      for (int k = 0; k < VEC; ++k) {
        float o = alpha * acc[k];
        o += beta * cp[k];
        cp[k] = o;
      }
    } else if (hints) {
#pragma unroll
      for (int k = 0; k < VEC; ++k) __stcs(cp + k, alpha * acc[k]);
    } else {
#pragma unroll
      for (int k = 0; k < VEC; ++k) cp[k] = alpha * acc[k];
    }
  }
}

template <typename T, int LPR>
static bsp_status launch_slab(const bsp_spmm_plan *p, const int32_t *ci, const void *val, const void *B,
                              int64_t ldb, int32_t col0, float *C, int64_t ldc, float *part, float a, float b,
                              int32_t hints, cudaStream_t s) {
  constexpr int G = 32 / LPR;
  const int64_t ntasks = p->nparts + (p->nshort + G - 1) / G;
  int64_t blocks = ceil_div(ntasks, 8);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_slab_kernel<T, LPR, SlabU<LPR>::U, SlabU<LPR>::UL><<<(unsigned)blocks, 256, 0, s>>>(
      p->nparts, reinterpret_cast<const int2 *>(p->long_se), p->nshort, p->short_rows,
      reinterpret_cast<const int2 *>(p->short_se), ci, (const T *)val, (const T *)B, ldb, col0, C, ldc, part, a, b,
      hints);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

// Slab width (columns per pass) for the slab engine; 0 when it cannot run
// (B rows not 16-byte aligned, N not a multiple of VEC).  With `want` == 0:
// the widest slab of at most 32 lanes of 16 bytes that divides N (graph
// 2^20, FP16, N = 256: 32 lanes 3.49 ms, 16 lanes in two passes 3.62).  Slabs
// sized so that B's slab stays in L2 measured slower (power-law graph 2^20,
// FP16, N = 128: four 32-column passes 2.42 ms against one 128-column pass
// 1.81 ms): the gathers run at the same rate from L2 as from DRAM, and every
// pass reads A again.
template <typename T>
static int slab_width(int32_t N, int32_t cols, const void *B, int64_t ldb, int32_t want) {
  constexpr int VEC = SpmmVec<T>::VEC;
  if ((uintptr_t)B % 16 != 0 || (ldb * (int64_t)sizeof(T)) % 16 != 0 || N % VEC != 0) return 0;
  if (want > 0) {
    if (want % VEC != 0 || N % want != 0) return -1;
    const int l = want / VEC;
    if (l > 32 || (l & (l - 1)) != 0) return -1;
    return want;
  }
  (void)cols;
  int l = 32;
  while (l > 1 && N % (l * VEC) != 0) l >>= 1;
  return l * VEC;
}

// The plan's L2 hints apply to slabs of B of at most kHintSlabBytes
// (cols x slab width), the size that stays in L2 during a pass; wider slabs
// gather with default caching (graph 2^20, FP16: hints at N = 32 (64 MB)
// 0.489 -> 0.473 ms, at N = 128 (one 268 MB slab) 1.822 -> 1.853 ms).
constexpr double kHintSlabBytes = 64.0 * 1024 * 1024;

template <typename T>
static bsp_status slab_typed(const bsp_spmm_plan *p, int32_t N, int32_t cols, int32_t ns, const int32_t *ci,
                             const void *val, const void *B, int64_t ldb, float *C, int64_t ldc, float *part,
                             float a, float b, cudaStream_t s) {
  constexpr int VEC = SpmmVec<T>::VEC;
  const int32_t hints = (double)cols * ns * sizeof(T) <= kHintSlabBytes ? p->slab_l2_hints : 0;
  for (int32_t col0 = 0; col0 < N; col0 += ns) {
    bsp_status st;
    switch (ns / VEC) {
      case 32: st = launch_slab<T, 32>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      case 16: st = launch_slab<T, 16>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      case 8: st = launch_slab<T, 8>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      case 4: st = launch_slab<T, 4>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      case 2: st = launch_slab<T, 2>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      case 1: st = launch_slab<T, 1>(p, ci, val, B, ldb, col0, C, ldc, part, a, b, hints, s); break;
      default: BSP_FAIL(BSP_ERR_UNSUPPORTED, "slab width");
    }
    BSP_TRY(st);
    BSP_TRY(split_reduce(p, ns, part, part + (int64_t)p->nparts * N, C + col0, ldc, a, b, s));
  }
  return BSP_OK;
}
}  // namespace bsp

extern "C" size_t bsp_spmm_plan_workspace(const bsp_spmm_plan *p, int32_t N) {
  return p ? ((size_t)p->nparts + (size_t)p->ngroups) * (size_t)(N > 0 ? N : 0) * sizeof(float) : 0;
}

namespace bsp {
static bsp_status spmm_planned_impl(const bsp_spmm_plan *p, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                    const int32_t *colIdx, const void *values, bsp_dtype dtype, const void *B,
                                    int32_t N, int64_t ldb, float *C, int64_t ldc, float alpha, float beta,
                                    void *workspace, size_t workspace_bytes, int32_t engine, int32_t slab_cols,
                                    cudaStream_t s);
}  // namespace bsp

extern "C" bsp_status bsp_spmm_csr_planned(const bsp_spmm_plan *p, int32_t cols, int32_t nnz,
                                           const int32_t *rowPtr, const int32_t *colIdx, const void *values,
                                           bsp_dtype dtype, const void *B, int32_t N, int64_t ldb, float *C,
                                           int64_t ldc, float alpha, float beta, void *workspace,
                                           size_t workspace_bytes, bsp_stream_t stream) {
  clear_error();
  return spmm_planned_impl(p, cols, nnz, rowPtr, colIdx, values, dtype, B, N, ldb, C, ldc, alpha, beta, workspace,
                           workspace_bytes, BSP_SPMM_AUTO, 0, as_stream(stream));
}

extern "C" bsp_status bsp_spmm_csr_planned_variant(const bsp_spmm_plan *p, int32_t cols, int32_t nnz,
                                                   const int32_t *rowPtr, const int32_t *colIdx,
                                                   const void *values, bsp_dtype dtype, const void *B, int32_t N,
                                                   int64_t ldb, float *C, int64_t ldc, float alpha, float beta,
                                                   void *workspace, size_t workspace_bytes, int32_t engine,
                                                   int32_t slab_cols, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(engine >= BSP_SPMM_AUTO && engine <= BSP_SPMM_SLAB, "unknown engine");
  BSP_CHECK_ARG(slab_cols >= 0, "negative slab width");
  return spmm_planned_impl(p, cols, nnz, rowPtr, colIdx, values, dtype, B, N, ldb, C, ldc, alpha, beta, workspace,
                           workspace_bytes, engine, slab_cols, as_stream(stream));
}

namespace bsp {
template <typename T>
static int slab_choice(const bsp_spmm_plan *p, int32_t N, int32_t cols, const void *B, int64_t ldb, int32_t engine,
                       int32_t slab_cols) {
  if (engine == BSP_SPMM_GROUPED) return 0;
  // automatic and explicit slab: the slab engine whenever it can run
  return slab_width<T>(N, cols, B, ldb, slab_cols);
}

static bsp_status spmm_planned_impl(const bsp_spmm_plan *p, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                    const int32_t *colIdx, const void *values, bsp_dtype dtype, const void *B,
                                    int32_t N, int64_t ldb, float *C, int64_t ldc, float alpha, float beta,
                                    void *workspace, size_t workspace_bytes, int32_t engine, int32_t slab_cols,
                                    cudaStream_t s) {
  BSP_CHECK_ARG(p && rowPtr && C, "null pointer");
  BSP_CHECK_ARG(N >= 0 && ldb >= N && ldc >= N, "bad N / leading dimensions");
  if (p->rows == 0 || N == 0) return BSP_OK;
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values && B), "null pointer");
  const size_t need = bsp_spmm_plan_workspace(p, N);
  BSP_CHECK_ARG(workspace_bytes >= need && (need == 0 || workspace), "workspace too small");
  float *part = reinterpret_cast<float *>(workspace);
  bsp_status st;
  int ns = 0;
  switch (dtype) {
    case BSP_F16: ns = slab_choice<__half>(p, N, cols, B, ldb, engine, slab_cols); break;
    case BSP_BF16: ns = slab_choice<__nv_bfloat16>(p, N, cols, B, ldb, engine, slab_cols); break;
    case BSP_F32: ns = slab_choice<float>(p, N, cols, B, ldb, engine, slab_cols); break;
    default: BSP_FAIL(BSP_ERR_UNSUPPORTED, "SpMM takes F16, BF16 or F32 values");
  }
  if (ns < 0 || (engine == BSP_SPMM_SLAB && ns == 0))
    BSP_FAIL(BSP_ERR_UNSUPPORTED, "the slab engine needs 16-byte aligned B rows and a slab width that is a power "
                                  "of two times 16 bytes dividing N");
  if (ns > 0) {
    if (nnz > 0 && !(colIdx && values && B)) BSP_FAIL(BSP_ERR_INVALID, "null pointer");
    switch (dtype) {
      case BSP_F16: return slab_typed<__half>(p, N, cols, ns, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
      case BSP_BF16:
        return slab_typed<__nv_bfloat16>(p, N, cols, ns, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
      default: return slab_typed<float>(p, N, cols, ns, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
    }
  }
  switch (dtype) {
    case BSP_F16:
      st = chunked_typed<__half>(p, N, rowPtr, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
      break;
    case BSP_BF16:
      st = chunked_typed<__nv_bfloat16>(p, N, rowPtr, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
      break;
    case BSP_F32:
      st = chunked_typed<float>(p, N, rowPtr, colIdx, values, B, ldb, C, ldc, part, alpha, beta, s);
      break;
    default:
      BSP_FAIL(BSP_ERR_UNSUPPORTED, "SpMM takes F16, BF16 or F32 values");
  }
  if (st != BSP_OK) return st;
  BSP_TRY(split_reduce(p, N, part, part + (int64_t)p->nparts * N, C, ldc, alpha, beta, s));
  return BSP_OK;
}
}  // namespace bsp

// ---------------------------------------------------------------------------
// Gathered-tile matrix (bsp_gtile): built on the host from host CSR arrays.
namespace bsp {
template <typename T>
static T host_cvt(double v);
template <> __half host_cvt<__half>(double v) { return __double2half(v); }
template <> __nv_bfloat16 host_cvt<__nv_bfloat16>(double v) { return __float2bfloat16_rn((float)v); }

template <typename T>
static bsp_status gtile_build(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rp, const int32_t *ci,
                              const double *val, bsp_gtile *g) {
  const int32_t ng = (rows + kTS - 1) / kTS;
  std::vector<int64_t> nch(ng + 1, 0);
  std::vector<std::vector<std::pair<int32_t, int32_t>>> ent(ng);   // (column, entry index) per group
#pragma omp parallel for schedule(dynamic, 64)
  for (int32_t gi = 0; gi < ng; ++gi) {
    auto &e = ent[gi];
    const int32_t r0 = gi * kTS, r1 = std::min(rows, r0 + kTS);
    e.reserve(rp[r1] - rp[r0]);
    for (int32_t k = rp[r0]; k < rp[r1]; ++k) e.push_back({ci[k], k});
    std::stable_sort(e.begin(), e.end(), [](const std::pair<int32_t, int32_t> &a, const std::pair<int32_t, int32_t> &b) {
      return a.first < b.first;
    });
    int64_t d = 0;
    for (size_t i = 0; i < e.size(); ++i)
      if (i == 0 || e[i].first != e[i - 1].first) ++d;
    nch[gi + 1] = (d + kTS - 1) / kTS;
  }
  for (int32_t gi = 0; gi < ng; ++gi) nch[gi + 1] += nch[gi];
  const int64_t nchunks = nch[ng];
  if (nchunks > INT32_MAX / 256) BSP_FAIL(BSP_ERR_UNSUPPORTED, "gathered tiles: too many chunks for int32 indexing");
  std::vector<int32_t> hcols((size_t)nchunks * kTS, 0);
  std::vector<T> htiles((size_t)nchunks * kTS * kTS, host_cvt<T>(0.0));
  // row of each entry: walk the group's rows
#pragma omp parallel for schedule(dynamic, 64)
  for (int32_t gi = 0; gi < ng; ++gi) {
    const auto &e = ent[gi];
    const int32_t r0 = gi * kTS;
    int64_t s = -1;
    for (size_t i = 0; i < e.size(); ++i) {
      if (i == 0 || e[i].first != e[i - 1].first) {
        ++s;
        hcols[(size_t)((nch[gi] + s / kTS) * kTS + s % kTS)] = e[i].first;
      }
      const int32_t k = e[i].second;
      // the entry's row: the last row of the group whose start is <= k
      int32_t r = r0;
      while (r + 1 < std::min(rows, r0 + kTS) && rp[r + 1] <= k) ++r;
      const int64_t chunk = nch[gi] + s / kTS;
      htiles[(size_t)chunk * kTS * kTS + tile_pos(r - r0, (int)(s % kTS))] = host_cvt<T>(val[k]);
    }
  }
  // pieces of up to kGtPieceChunks chunks; groups with several get partial slots
  std::vector<int32_t> pptr{0}, pgroup, pslot, gpiece(ng + 1, 0), split;
  int32_t slots = 0;
  for (int32_t gi = 0; gi < ng; ++gi) {
    const int64_t c0 = nch[gi], c1 = nch[gi + 1];
    const int64_t np = std::max<int64_t>(1, (c1 - c0 + kGtPieceChunks - 1) / kGtPieceChunks);
    if (np > 1) split.push_back(gi);
    for (int64_t p = 0; p < np; ++p) {
      pptr.push_back((int32_t)std::min(c1, c0 + (p + 1) * kGtPieceChunks));
      pgroup.push_back(gi);
      pslot.push_back(np > 1 ? slots++ : -1);
    }
    gpiece[gi + 1] = (int32_t)pgroup.size();
  }
  bsp_gtile o{};
  o.rows = rows;
  o.cols = cols;
  o.nnz = nnz;
  o.dtype = std::is_same<T, __half>::value ? BSP_F16 : BSP_BF16;
  o.nchunks = nchunks;
  o.ngroups = ng;
  o.npieces = (int32_t)pgroup.size();
  o.nsplit = (int32_t)split.size();
  o.nslots = slots;
  cudaStream_t s = 0;
  auto up = [&](auto **dst, const auto &v) -> bsp_status {
    using E = typename std::remove_reference<decltype(v)>::type::value_type;
    E *p = nullptr;
    BSP_TRY(dalloc(&p, std::max<size_t>(1, v.size()), s));
    if (!v.empty()) BSP_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice, s));
    *dst = reinterpret_cast<typename std::remove_pointer<decltype(dst)>::type>(p);
    return BSP_OK;
  };
  bsp_status st = up(&o.piece_ptr, pptr);
  if (st == BSP_OK) st = up(&o.piece_group, pgroup);
  if (st == BSP_OK) st = up(&o.piece_slot, pslot);
  if (st == BSP_OK) st = up(&o.group_piece, gpiece);
  if (st == BSP_OK) st = up(&o.split_groups, split);
  if (st == BSP_OK) st = up(&o.chunk_cols, hcols);
  T *tiles = nullptr;
  if (st == BSP_OK) st = up(&tiles, htiles);
  o.chunk_tiles = tiles;
  if (st == BSP_OK) st = dalloc(&o.err, 1, s);
  if (st == BSP_OK && cudaMemsetAsync(o.err, 0, sizeof(int32_t), s) != cudaSuccess) st = BSP_ERR_CUDA;
  if (st == BSP_OK && cudaStreamSynchronize(s) != cudaSuccess) st = BSP_ERR_CUDA;   // host vectors go away
  *g = o;
  return st;
}
}  // namespace bsp

extern "C" bsp_status bsp_gtile_free(bsp_gtile *g) {
  clear_error();
  if (!g) return BSP_OK;
  cudaStream_t s = 0;
  dfree(g->piece_ptr, s);
  dfree(g->piece_group, s);
  dfree(g->piece_slot, s);
  dfree(g->group_piece, s);
  dfree(g->split_groups, s);
  dfree(g->chunk_cols, s);
  if (g->chunk_tiles) cudaFreeAsync(g->chunk_tiles, s);
  g->chunk_tiles = nullptr;
  dfree(g->err, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_gtile_create_host(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                            const int32_t *colIdx, const double *values, bsp_dtype dtype,
                                            bsp_gtile *out) {
  clear_error();
  BSP_CHECK_ARG(out && rowPtr && rows >= 0 && cols >= 0 && nnz >= 0, "bad argument");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values), "null pointer");
  BSP_CHECK_ARG(dtype == BSP_F16 || dtype == BSP_BF16, "gathered tiles are F16 or BF16");
  BSP_CHECK_ARG(rowPtr[0] == 0 && rowPtr[rows] == nnz, "rowPtr[0] must be 0 and rowPtr[rows] == nnz");
  *out = bsp_gtile{};
  bsp_status st = dtype == BSP_F16 ? gtile_build<__half>(rows, cols, nnz, rowPtr, colIdx, values, out)
                                   : gtile_build<__nv_bfloat16>(rows, cols, nnz, rowPtr, colIdx, values, out);
  if (st != BSP_OK) bsp_gtile_free(out);
  return st;
}

extern "C" size_t bsp_gtile_workspace(const bsp_gtile *g, int32_t N) {
  return g ? (size_t)g->nslots * kTS * (size_t)(N > 0 ? N : 0) * sizeof(float) : 0;
}

extern "C" bsp_status bsp_gtile_spmm(const bsp_gtile *g, const void *B, int32_t N, int64_t ldb, float *C,
                                     int64_t ldc, float alpha, float beta, void *workspace, size_t workspace_bytes,
                                     bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(g && B && C, "null pointer");
  BSP_CHECK_ARG(N > 0 && N % 8 == 0, "N must be a positive multiple of 8");
  BSP_CHECK_ARG(ldb >= N && ldc >= N, "leading dimension smaller than N");
  BSP_CHECK_ARG((uintptr_t)B % 16 == 0 && (ldb * 2) % 16 == 0, "B must be 16-byte aligned with ldb % 8 == 0");
  const size_t need = bsp_gtile_workspace(g, N);
  BSP_CHECK_ARG(workspace_bytes >= need && (need == 0 || workspace), "workspace too small");
  if (g->ngroups == 0) return BSP_OK;
  cudaStream_t s = as_stream(stream);
  const int32_t W = N >= 128 ? 128 : 64;
  // one launch per slab of W columns, as the block kernel's (smat_spmm_tcp),
  // or all slabs in one launch
  const int32_t per = kGtcPerSlab ? 1 : (int32_t)ceil_div(N, W);
  const int64_t total = (int64_t)g->npieces * per;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(total, (int64_t)sm_count() * 8));
  float *part = static_cast<float *>(workspace);
  for (int32_t c0 = 0; c0 < N; c0 += W * per) {
    if (g->dtype == BSP_F16)
      spmm_gtc_kernel<__half><<<grid, kTcpThreads, kGtcSmem, s>>>(
          g->rows, N, W, c0, per, g->npieces, g->piece_ptr, g->piece_group, g->piece_slot, g->chunk_cols,
          (const __half *)g->chunk_tiles, (const __half *)B, ldb, C, ldc, part, alpha, beta, g->err);
    else
      spmm_gtc_kernel<__nv_bfloat16><<<grid, kTcpThreads, kGtcSmem, s>>>(
          g->rows, N, W, c0, per, g->npieces, g->piece_ptr, g->piece_group, g->piece_slot, g->chunk_cols,
          (const __nv_bfloat16 *)g->chunk_tiles, (const __nv_bfloat16 *)B, ldb, C, ldc, part, alpha, beta,
          g->err);
  }
  BSP_LAUNCH_CHECK();
  if (g->nsplit > 0) {
    const int64_t work = (int64_t)g->nsplit * kTS * N;
    const unsigned rg = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(work, 256), (int64_t)sm_count() * 16));
    gtile_reduce_kernel<<<rg, 256, 0, s>>>(g->nsplit, g->split_groups, g->group_piece, g->piece_slot, g->rows, N,
                                           part, C, ldc, alpha, beta);
    BSP_LAUNCH_CHECK();
  }
  return BSP_OK;
}

extern "C" bsp_status bsp_gtile_check(const bsp_gtile *g, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(g, "null pointer");
  int32_t h = 0;
  cudaStream_t s = as_stream(stream);
  BSP_CUDA(cudaMemcpyAsync(&h, g->err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  if (h) BSP_FAIL(BSP_ERR_TIMEOUT, "a bounded wait of the gathered-tile kernel gave up");
  return BSP_OK;
}
