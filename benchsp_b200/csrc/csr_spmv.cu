// CSR SpMV kernels for sm_100a.
//
// Replaces the reference's CSR paths:
//   spmv_fp64 (thread per row)            src/csrspmv.cu:39-57
//   spmv_fp64_balance (16-nnz chunks, atomics) src/csrspmv.cu:84-102
//   spmv_fp16/fp64 + *_long (row split at 128 nnz) src/spmv.cu:13-107
// with three deterministic kernels (no atomics, each y element written by
// exactly one thread except the merge-path carry fix-up, which runs after):
//   * scalar: one thread per row, left-to-right sum with separately rounded
//     multiply and add -- bit-identical to ref_spmv_fp64 / ref_spmv_fp16
//     (src/ref.cpp:3-37) on the same inputs;
//   * vector: a power-of-two group of lanes per row, strided loads of
//     values/columns, read-only cached gathers of x, shuffle reduction;
//   * merge-path: every warp takes an equal share of (rows + nnz) merge
//     items, so power-law rows cost the same as short ones; warp-level
//     segmented scan plus a carry fix-up kernel over a small workspace.
#include "bsp_internal.cuh"

namespace bsp {

template <typename V> struct AccOf { using T = float; };
template <> struct AccOf<double> { using T = double; };

template <typename V> __device__ __forceinline__ typename AccOf<V>::T to_acc(V v);
template <> __device__ __forceinline__ double to_acc<double>(double v) { return v; }
template <> __device__ __forceinline__ float to_acc<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_acc<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_acc<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename V> __device__ __forceinline__ V from_acc(typename AccOf<V>::T v);
template <> __device__ __forceinline__ double from_acc<double>(double v) { return v; }
template <> __device__ __forceinline__ float from_acc<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_acc<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

template <typename V, typename A>
__device__ __forceinline__ void store_y(V *y, int64_t i, A sum, A alpha, A beta) {
  A r = alpha * sum;
  if (beta != A(0)) r += beta * to_acc<V>(y[i]);
  y[i] = from_acc<V>(r);
}

// One thread per row, sum in column order with no fused multiply-add: the
// exact operation sequence of ref_spmv_fp64/ref_spmv_fp16 (src/ref.cpp).
template <typename V>
__global__ void __launch_bounds__(256) csr_scalar_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                                         const int32_t *__restrict__ colIdx,
                                                         const V *__restrict__ val, const V *__restrict__ x,
                                                         V *__restrict__ y, typename AccOf<V>::T alpha,
                                                         typename AccOf<V>::T beta) {
  using A = typename AccOf<V>::T;
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    A sum = A(0);
    const int32_t e = rowPtr[r + 1];
    for (int32_t j = rowPtr[r]; j < e; ++j)
      sum = add_rn(sum, mul_rn(to_acc<V>(val[j]), to_acc<V>(__ldg(&x[colIdx[j]]))));
    if (alpha == A(1) && beta == A(0))
      y[r] = from_acc<V>(sum);
    else
      store_y<V, A>(y, r, sum, alpha, beta);
  }
}

constexpr int kWarpRowFactor = 64;

// LPR lanes per row (LPR in {1,2,4,8,16,32}); grid-stride over rows.
template <typename V, int LPR>
__global__ void __launch_bounds__(256) csr_vector_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                                         const int32_t *__restrict__ colIdx,
                                                         const V *__restrict__ val, const V *__restrict__ x,
                                                         V *__restrict__ y, typename AccOf<V>::T alpha,
                                                         typename AccOf<V>::T beta) {
  using A = typename AccOf<V>::T;
  const int sub = threadIdx.x & (LPR - 1);
  const int64_t groups = (int64_t)gridDim.x * (blockDim.x / LPR);
  // The loop bound is uniform across the warp (base is the warp's first row)
  // so the shuffle reduction always runs with every lane present.
  const int64_t warp_first = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LPR;
  for (int64_t base = warp_first; base < rows; base += groups) {
    const int64_t r = base + (threadIdx.x & 31) / LPR;
    const bool active = r < rows;
    const int32_t s = active ? rowPtr[r] : 0, e0 = active ? rowPtr[r + 1] : 0;
    // rows longer than kWarpRowFactor entries per lane are summed by the
    // whole warp after the pass, so one long row does not hold its warp's
    // other rows (power-law rows at one lane per row)
    const bool big = LPR < 32 && e0 - s > kWarpRowFactor * LPR;
    const int32_t e = big ? s : e0;
    // The first kFirst entries of each lane are loaded together, then their x
    // gathers together: the rowPtr -> column -> x chain is paid once per
    // kFirst entries instead of once per entry.
    constexpr int kFirst = LPR == 1 ? 8 : 4;
    int32_t c[kFirst];
    V a[kFirst];
#pragma unroll
    for (int k = 0; k < kFirst; ++k) {
      const int32_t j = s + sub + k * LPR;
      c[k] = j < e ? colIdx[j] : -1;
      a[k] = j < e ? val[j] : V(0);
    }
    A sum = A(0);
#pragma unroll
    for (int k = 0; k < kFirst; ++k)
      if (c[k] >= 0) sum = fma(to_acc<V>(a[k]), to_acc<V>(__ldg(&x[c[k]])), sum);
#pragma unroll 4
    for (int32_t j = s + sub + kFirst * LPR; j < e; j += LPR)
      sum = fma(to_acc<V>(val[j]), to_acc<V>(__ldg(&x[colIdx[j]])), sum);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, LPR);
    if (active && sub == 0 && !big) store_y<V, A>(y, r, sum, alpha, beta);
    if constexpr (LPR < 32) {
      unsigned todo = __ballot_sync(0xffffffffu, big && sub == 0);
      const int lane = threadIdx.x & 31;
      while (todo) {   // warp-uniform
        const int b = __ffs(todo) - 1;
        todo &= todo - 1;
        const int64_t br = base + b / LPR;
        const int32_t bs = rowPtr[br], be = rowPtr[br + 1];
        A ws = A(0);
        int32_t j = bs + lane;
        for (; j + 96 < be; j += 128) {
          int32_t c[4];
          V a[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            c[u] = colIdx[j + 32 * u];
            a[u] = val[j + 32 * u];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) ws = fma(to_acc<V>(a[u]), to_acc<V>(__ldg(&x[c[u]])), ws);
        }
        for (; j < be; j += 32) ws = fma(to_acc<V>(val[j]), to_acc<V>(__ldg(&x[colIdx[j]])), ws);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ws += __shfl_xor_sync(0xffffffffu, ws, o);
        if (lane == 0) store_y<V, A>(y, br, ws, alpha, beta);
      }
    }
  }
}

// Warp per 32 consecutive rows ("stream").  The warp's nonzero range
// [rowPtr[r0], rowPtr[r0+32]) is read in pieces of kStreamPiece entries:
// every lane loads kStreamPiece/32 values and column indices (one coalesced
// 256-byte access per array and step), issues their x gathers together and
// stores the products to shared memory; then each lane adds its own row's
// products of the piece left to right.  Every row costs the same dependent
// chain (rowPtr -> entries -> x) as in the thread-per-row kernel, but the
// entry loads are coalesced and all of a piece's gathers are in flight at
// once.  Multiply and add are rounded separately in column order, so the
// result equals csr_scalar_kernel's (and ref_spmv_fp64's) bit for bit.
constexpr int kStreamPiece = 256;
constexpr int kStreamThreads = 256;

// 48 registers (5 CTAs per SM).  Capped at 40 / 32 registers it measured
// 16.7 / 17.3 us against 16.5 us on the 7-point Poisson 64^3 (L2 flushed).
template <typename V>
__global__ void __launch_bounds__(kStreamThreads) csr_stream_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                                                    const int32_t *__restrict__ colIdx,
                                                                    const V *__restrict__ val,
                                                                    const V *__restrict__ x, V *__restrict__ y,
                                                                    typename AccOf<V>::T alpha,
                                                                    typename AccOf<V>::T beta) {
  using A = typename AccOf<V>::T;
  constexpr int K = kStreamPiece / 32;
  __shared__ A prod[kStreamThreads / 32][kStreamPiece];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  A *pw = prod[wib];
  const int64_t nblk = ((int64_t)rows + 31) / 32;
  const int64_t nwarps = (int64_t)gridDim.x * (kStreamThreads / 32);
  for (int64_t wb = (int64_t)blockIdx.x * (kStreamThreads / 32) + wib; wb < nblk; wb += nwarps) {
    const int64_t r = wb * 32 + lane;
    const bool active = r < rows;
    const int32_t rs = active ? rowPtr[r] : 0, re = active ? rowPtr[r + 1] : 0;
    const int32_t base = __shfl_sync(0xffffffffu, rs, 0);
    const int64_t last = min((int64_t)rows, wb * 32 + 32) - 1 - wb * 32;   // last active lane
    const int32_t end = __shfl_sync(0xffffffffu, re, (int)last);
    A sum = A(0);
    for (int32_t pb = base; pb < end; pb += kStreamPiece) {   // warp-uniform
      int32_t c[K];
      V a[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int32_t j = pb + k * 32 + lane;
        c[k] = j < end ? colIdx[j] : -1;
        a[k] = j < end ? val[j] : V(0);
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (c[k] >= 0) pw[k * 32 + lane] = mul_rn(to_acc<V>(a[k]), to_acc<V>(__ldg(&x[c[k]])));
      __syncwarp();
      const int32_t lo = rs > pb ? rs : pb;
      const int32_t hi = re < pb + kStreamPiece ? re : pb + kStreamPiece;
      for (int32_t j = lo; j < hi; ++j) sum = add_rn(sum, pw[j - pb]);
      __syncwarp();
    }
    if (active) {
      if (alpha == A(1) && beta == A(0))
        y[r] = from_acc<V>(sum);
      else
        store_y<V, A>(y, r, sum, alpha, beta);
    }
  }
}

// ---------------------------------------------------------------------------
// Merge-path SpMV (FP64).  Merge items are the rows' end offsets
// (rowPtr[1..rows]) interleaved with the nnz indices 0..nnz-1; every thread
// consumes kItems consecutive items.  Path coordinate (i, j) = (rows
// finished, nnz consumed); a row-end item is taken before nnz item j when
// rowPtr[i+1] <= j.
constexpr int kMergeItems = 8;
constexpr int kMergeThreads = 256;
constexpr int kMergeWarpItems = kWarp * kMergeItems;

__device__ __forceinline__ void merge_path_search(int64_t diag, const int32_t *__restrict__ rowEnd,
                                                  int32_t rows, int32_t nnz, int32_t &i, int32_t &j) {
  int64_t lo = diag - nnz > 0 ? diag - nnz : 0;
  int64_t hi = diag < rows ? diag : rows;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if ((int64_t)rowEnd[mid] <= diag - mid - 1)
      lo = mid + 1;
    else
      hi = mid;
  }
  i = (int32_t)lo;
  j = (int32_t)(diag - lo);
}

// Per-warp carry: the partial sum of the row a warp's range ends inside.
// carry_row = -1 when the warp ends exactly on a row boundary.
__global__ void __launch_bounds__(kMergeThreads) csr_merge_kernel(
    int32_t rows, int32_t nnz, const int32_t *__restrict__ rowPtr, const int32_t *__restrict__ colIdx,
    const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y, double alpha,
    double beta, int32_t *__restrict__ carry_row, double *__restrict__ carry_val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * kMergeThreads + threadIdx.x) >> 5;
  const int64_t total = (int64_t)rows + nnz;
  const int64_t warp_begin = warp * kMergeWarpItems;
  if (warp_begin >= total) return;  // whole warp exits together
  const int64_t diag = warp_begin + (int64_t)lane * kMergeItems;
  const int64_t diag_end = diag + kMergeItems < total ? diag + kMergeItems : total;

  int32_t i = 0, j = 0;
  if (diag < total) merge_path_search(diag, rowPtr + 1, rows, nnz, i, j);

  double acc = 0.0;
  int32_t first_row = -1;  // first row that ends in this lane's range
  double first_val = 0.0;
  for (int64_t d = diag; d < diag_end; ++d) {
    if (i < rows && rowPtr[i + 1] <= j) {
      if (first_row < 0) {
        first_row = i;
        first_val = acc;
      } else {
        double r = alpha * acc;
        if (beta != 0.0) r += beta * y[i];
        y[i] = r;
      }
      acc = 0.0;
      ++i;
    } else {
      acc = fma(val[j], __ldg(&x[colIdx[j]]), acc);
      ++j;
    }
  }
  // Segmented inclusive scan of the lanes' trailing partials: a lane that
  // finished a row starts a new segment.
  const bool head = first_row >= 0;
  double seg = acc;
  bool seg_head = head;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double v = __shfl_up_sync(0xffffffffu, seg, o);
    bool h = __shfl_up_sync(0xffffffffu, seg_head, o);
    if (lane >= o && !seg_head) {
      seg += v;
      seg_head = h;
    }
  }
  // carry_in for this lane = inclusive result of lane-1.
  double carry_in = __shfl_up_sync(0xffffffffu, seg, 1);
  if (lane == 0) carry_in = 0.0;
  if (head) {
    double r = alpha * (first_val + carry_in);
    if (beta != 0.0) r += beta * y[first_row];
    y[first_row] = r;
  }
  if (lane == 31) {
    // Row the warp ends inside (i after the last lane's items), if unfinished.
    const int64_t wend = warp_begin + kMergeWarpItems < total ? warp_begin + kMergeWarpItems : total;
    int32_t ei, ej;
    merge_path_search(wend, rowPtr + 1, rows, nnz, ei, ej);
    const bool open = ei < rows && ej > rowPtr[ei];
    carry_row[warp] = open ? ei : -1;
    carry_val[warp] = open ? seg : 0.0;
  }
}

// Adds the carries to the rows they belong to.  Carries are ordered by row;
// the first carry of each run of equal rows sums the run (deterministic).
__global__ void csr_merge_fixup_kernel(int64_t nwarps, const int32_t *__restrict__ carry_row,
                                       const double *__restrict__ carry_val, double *__restrict__ y,
                                       double alpha) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwarps;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int32_t r = carry_row[w];
    if (r < 0) continue;
    if (w > 0 && carry_row[w - 1] == r) continue;
    double s = 0.0;
    for (int64_t k = w; k < nwarps && carry_row[k] == r; ++k) s += carry_val[k];
    y[r] += alpha * s;
  }
}

static int64_t merge_warps(int32_t rows, int32_t nnz) {
  return ceil_div((int64_t)rows + nnz, kMergeWarpItems);
}

bsp_status launch_merge(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                        const double *val, const double *x, double *y, double alpha, double beta,
                        int32_t *carry_row, double *carry_val, cudaStream_t s) {
  const int64_t nw = merge_warps(rows, nnz);
  if (nw == 0) return BSP_OK;
  const int64_t blocks = ceil_div(nw * kWarp, kMergeThreads);
  csr_merge_kernel<<<(unsigned)blocks, kMergeThreads, 0, s>>>(rows, nnz, rowPtr, colIdx, val, x, y, alpha,
                                                              beta, carry_row, carry_val);
  BSP_LAUNCH_CHECK();
  const int64_t fb = ceil_div(nw, 256);
  csr_merge_fixup_kernel<<<(unsigned)(fb < 4096 ? fb : 4096), 256, 0, s>>>(nw, carry_row, carry_val, y, alpha);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

size_t merge_workspace_bytes(int32_t rows, int32_t nnz) {
  const int64_t nw = merge_warps(rows, nnz);
  const size_t rows_b = ((size_t)nw * sizeof(int32_t) + 255) & ~size_t(255);
  return rows_b + (size_t)nw * sizeof(double);
}

// ---------------------------------------------------------------------------
template <typename V>
static bsp_status launch_vector(int lpr, int32_t rows, const int32_t *rp, const int32_t *ci, const V *v,
                                const V *x, V *y, typename AccOf<V>::T a, typename AccOf<V>::T b,
                                cudaStream_t s) {
  const int threads = 256;
  const int64_t rows_per_block = threads / lpr;
  int64_t blocks = ceil_div(rows, rows_per_block);
  const int64_t cap = (int64_t)sm_count() * 64;  // grid-stride beyond this
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  switch (lpr) {
#define BSP_VEC_CASE(L)                                                                    \
  case L:                                                                                  \
    csr_vector_kernel<V, L><<<(unsigned)blocks, threads, 0, s>>>(rows, rp, ci, v, x, y, a, b); \
    break;
    BSP_VEC_CASE(1) BSP_VEC_CASE(2) BSP_VEC_CASE(4) BSP_VEC_CASE(8) BSP_VEC_CASE(16) BSP_VEC_CASE(32)
#undef BSP_VEC_CASE
    default:
      BSP_FAIL(BSP_ERR_INVALID, "lanes_per_row must be a power of two in [1,32]");
  }
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename V>
static bsp_status launch_scalar(int32_t rows, const int32_t *rp, const int32_t *ci, const V *v, const V *x,
                                V *y, typename AccOf<V>::T a, typename AccOf<V>::T b, cudaStream_t s) {
  int64_t blocks = ceil_div(rows, 256);
  const int64_t cap = (int64_t)sm_count() * 64;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  csr_scalar_kernel<V><<<(unsigned)blocks, 256, 0, s>>>(rows, rp, ci, v, x, y, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

template <typename V>
static bsp_status launch_stream(int32_t rows, const int32_t *rp, const int32_t *ci, const V *v, const V *x, V *y,
                                typename AccOf<V>::T a, typename AccOf<V>::T b, cudaStream_t s) {
  const int64_t warps = ceil_div(rows, 32);
  int64_t blocks = ceil_div(warps, kStreamThreads / 32);
  const int64_t cap = (int64_t)sm_count() * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  csr_stream_kernel<V><<<(unsigned)blocks, kStreamThreads, 0, s>>>(rows, rp, ci, v, x, y, a, b);
  BSP_LAUNCH_CHECK();
  return BSP_OK;
}

// Lanes per row from the mean row length: one lane per row up to 8 entries
// (those are loaded together), then the smallest power of two >= mean/4,
// up to 32.
int auto_lanes(int32_t rows, int32_t nnz) {
  const double mean = rows > 0 ? (double)nnz / rows : 0.0;
  if (mean <= 8.0) return 1;
  int l = 2;
  while (l < 32 && 4.0 * l < mean) l <<= 1;
  return l;
}

template <typename V>
static bsp_status csr_dispatch(int32_t rows, int32_t nnz, const int32_t *rp, const int32_t *ci, const V *v,
                               const V *x, V *y, double alpha, double beta, int32_t algo, int32_t lpr,
                               cudaStream_t s) {
  using A = typename AccOf<V>::T;
  if (algo == BSP_CSR_SCALAR) return launch_scalar<V>(rows, rp, ci, v, x, y, (A)alpha, (A)beta, s);
  if (algo == BSP_CSR_STREAM) return launch_stream<V>(rows, rp, ci, v, x, y, (A)alpha, (A)beta, s);
  if (lpr <= 0) lpr = auto_lanes(rows, nnz);
  return launch_vector<V>(lpr, rows, rp, ci, v, x, y, (A)alpha, (A)beta, s);
}

}  // namespace bsp

using namespace bsp;

extern "C" size_t bsp_csr_merge_workspace(int32_t rows, int32_t nnz) {
  return merge_workspace_bytes(rows, nnz);
}

extern "C" bsp_status bsp_csr_spmv_merge_f64(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                             const int32_t *colIdx, const double *values, const double *x,
                                             double *y, double alpha, double beta, void *workspace,
                                             size_t workspace_bytes, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  if (rows == 0) return BSP_OK;
  BSP_CHECK_ARG(rowPtr && y, "null pointer");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values && x), "null pointer");
  const size_t need = merge_workspace_bytes(rows, nnz);
  BSP_CHECK_ARG(workspace && workspace_bytes >= need, "workspace too small");
  BSP_CHECK_ARG(((uintptr_t)workspace & 15) == 0, "workspace must be 16-byte aligned");
  const int64_t nw = ceil_div((int64_t)rows + nnz, kMergeWarpItems);
  int32_t *carry_row = reinterpret_cast<int32_t *>(workspace);
  double *carry_val = reinterpret_cast<double *>(reinterpret_cast<char *>(workspace) +
                                                 (((size_t)nw * sizeof(int32_t) + 255) & ~size_t(255)));
  return launch_merge(rows, nnz, rowPtr, colIdx, values, x, y, alpha, beta, carry_row, carry_val,
                      as_stream(stream));
}

extern "C" bsp_status bsp_csr_spmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                   const int32_t *colIdx, const void *values, bsp_dtype dtype, const void *x,
                                   void *y, double alpha, double beta, int32_t algo, int32_t lanes_per_row,
                                   bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  if (rows == 0) return BSP_OK;
  BSP_CHECK_ARG(rowPtr && y, "null pointer");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values && x), "null pointer");
  BSP_CHECK_ARG(lanes_per_row >= 0 && lanes_per_row <= 32 && (lanes_per_row & (lanes_per_row - 1)) == 0,
                "lanes_per_row must be 0 or a power of two <= 32");
  cudaStream_t s = as_stream(stream);
  if (algo == BSP_CSR_MERGE) {
    BSP_CHECK_ARG(dtype == BSP_F64, "merge-path is FP64 only");
    const size_t need = merge_workspace_bytes(rows, nnz);
    void *ws = nullptr;
    BSP_CUDA(cudaMallocAsync(&ws, need, s));
    bsp_status st = bsp_csr_spmv_merge_f64(rows, cols, nnz, rowPtr, colIdx, (const double *)values,
                                           (const double *)x, (double *)y, alpha, beta, ws, need, stream);
    cudaFreeAsync(ws, s);
    return st;
  }
  if (algo == BSP_CSR_AUTO) {
    // Irregular rows (max far above mean) go through merge-path; the row
    // statistics are not known here without a pass, so AUTO means VECTOR
    // with lanes from the mean.  Plans pick MERGE from measured features.
    algo = BSP_CSR_VECTOR;
  }
  BSP_CHECK_ARG(algo == BSP_CSR_VECTOR || algo == BSP_CSR_SCALAR || algo == BSP_CSR_STREAM, "unknown algo");
  switch (dtype) {
    case BSP_F64:
      return csr_dispatch<double>(rows, nnz, rowPtr, colIdx, (const double *)values, (const double *)x,
                                  (double *)y, alpha, beta, algo, lanes_per_row, s);
    case BSP_F32:
      return csr_dispatch<float>(rows, nnz, rowPtr, colIdx, (const float *)values, (const float *)x,
                                 (float *)y, alpha, beta, algo, lanes_per_row, s);
    case BSP_F16:
      return csr_dispatch<__half>(rows, nnz, rowPtr, colIdx, (const __half *)values, (const __half *)x,
                                  (__half *)y, alpha, beta, algo, lanes_per_row, s);
    case BSP_BF16:
      return csr_dispatch<__nv_bfloat16>(rows, nnz, rowPtr, colIdx, (const __nv_bfloat16 *)values,
                                         (const __nv_bfloat16 *)x, (__nv_bfloat16 *)y, alpha, beta, algo,
                                         lanes_per_row, s);
  }
  BSP_FAIL(BSP_ERR_INVALID, "unknown dtype");
}
