// FP64 SpMV format autotuner and tuned executor.
//
// Model mode (no conversion): from the row-length statistics and the exact
// number of 4x4 and 8x8 blocks, compare bytes per nonzero scaled by the
// efficiency each kernel reached on the B200:
//   CSR vector  (8 + 4) B / nnz                at ~0.7 of the copy bandwidth
//   BSR bs x bs (8 bs^2 + 4) / (bs^2 fill) B   at ~1.05
// and send skewed matrices (a row of >= 256 nonzeros and max > 32 x mean)
// to DASP, whose layout balances long rows.  Measure mode converts to every
// candidate that can pay off (BSR only when its fill is at least 0.3, DASP
// only with rows of >= 32 nonzeros), times 10 SpMVs of each and keeps the
// fastest.  Choices are cached by a structural hash of the matrix.
#include <stdio.h>
#include <stdlib.h>

#include <cmath>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

struct RowStats {
  unsigned long long sum_sq;
  unsigned long long long_rows;
  int max_len;
  int pad;
};

__global__ void row_stats_kernel(int32_t rows, const int32_t *__restrict__ rowPtr, RowStats *__restrict__ out) {
  unsigned long long sq = 0, lr = 0;
  int mx = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    const int len = rowPtr[r + 1] - rowPtr[r];
    sq += (unsigned long long)len * (unsigned long long)len;
    lr += len >= 256;
    mx = max(mx, len);
  }
  for (int o = 16; o > 0; o >>= 1) {
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
    lr += __shfl_xor_sync(0xffffffffu, lr, o);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out->sum_sq, sq);
    atomicAdd(&out->long_rows, lr);
    atomicMax(&out->max_len, mx);
  }
}

// Distinct bs x bs blocks: one thread per block-row walks its bs sorted rows
// in step (a bs-way merge on col / bs).
template <int BS>
__global__ void block_count_kernel(int32_t rows, const int32_t *__restrict__ rowPtr,
                                   const int32_t *__restrict__ colIdx, unsigned long long *__restrict__ out) {
  unsigned long long cnt = 0;
  const int64_t brows = (rows + BS - 1) / BS;
  for (int64_t br = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; br < brows; br += (int64_t)gridDim.x * blockDim.x) {
    int32_t p[BS], e[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) {
      const int64_t r = br * BS + k;
      p[k] = r < rows ? rowPtr[r] : 0;
      e[k] = r < rows ? rowPtr[r + 1] : 0;
    }
    for (;;) {
      int32_t m = INT32_MAX;
#pragma unroll
      for (int k = 0; k < BS; ++k)
        if (p[k] < e[k]) m = min(m, colIdx[p[k]] / BS);
      if (m == INT32_MAX) break;
      ++cnt;
#pragma unroll
      for (int k = 0; k < BS; ++k)
        while (p[k] < e[k] && colIdx[p[k]] / BS == m) ++p[k];
    }
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, cnt);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Order-sensitive structural hash: a wrapping sum of mix(position, value)
// over rowPtr and colIdx (deterministic whatever the thread order).
__global__ void key_kernel(int32_t rows, int32_t nnz, const int32_t *__restrict__ rowPtr,
                           const int32_t *__restrict__ colIdx, unsigned long long *__restrict__ out) {
  unsigned long long h = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= rows; i += stride)
    h += mix64(((unsigned long long)i << 32) ^ (unsigned)rowPtr[i] ^ 0x5bd1e995ull);
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += stride)
    h += mix64(((unsigned long long)j << 32) ^ (unsigned)colIdx[j] ^ 0x27d4eb2full);
  for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

int auto_lanes(int32_t rows, int32_t nnz);  // csr_spmv.cu

namespace {

std::mutex g_mu;
std::unordered_map<uint64_t, bsp_tune_result> g_cache;
bool g_file_loaded = false;

const char *cache_path() { return getenv("BSP_TUNE_CACHE"); }

void load_file_locked() {
  if (g_file_loaded) return;
  g_file_loaded = true;
  const char *p = cache_path();
  if (!p) return;
  FILE *f = fopen(p, "r");
  if (!f) return;
  unsigned long long key;
  bsp_tune_result r{};
  while (fscanf(f, "%llx %d %d %d %d %d %lf", &key, &r.format, &r.csr_algo, &r.lanes, &r.bs, &r.bsr_algo,
                &r.spmv_us) == 7) {
    r.key = key;
    g_cache[key] = r;
  }
  fclose(f);
}

void append_file_locked(const bsp_tune_result &r) {
  const char *p = cache_path();
  if (!p) return;
  FILE *f = fopen(p, "a");
  if (!f) return;
  fprintf(f, "%016llx %d %d %d %d %d %.3f\n", (unsigned long long)r.key, r.format, r.csr_algo, r.lanes, r.bs,
          r.bsr_algo, r.spmv_us);
  fclose(f);
}

unsigned grid_for(int64_t n) {
  int64_t g = ceil_div(n > 0 ? n : 1, 256);
  const int64_t cap = (int64_t)sm_count() * 16;
  return (unsigned)(g > cap ? cap : g);
}

}  // namespace

bsp_status matrix_key(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx, int32_t cols,
                      uint64_t *key, cudaStream_t s) {
  unsigned long long *d = nullptr;
  BSP_TRY(dalloc(&d, 1, s));
  BSP_CUDA(cudaMemsetAsync(d, 0, sizeof(*d), s));
  key_kernel<<<grid_for((int64_t)rows + nnz), 256, 0, s>>>(rows, nnz, rowPtr, colIdx, d);
  BSP_LAUNCH_CHECK();
  unsigned long long h = 0;
  BSP_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  dfree(d, s);
  // fold in the sizes
  h ^= (unsigned long long)rows * 0x9E3779B97F4A7C15ull;
  h ^= ((unsigned long long)cols << 21) * 0xBF58476D1CE4E5B9ull;
  h ^= ((unsigned long long)nnz << 42) ^ ((unsigned long long)nnz >> 22);
  *key = h;
  return BSP_OK;
}

static bsp_status stats(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                        bsp_tune_result &r, cudaStream_t s) {
  RowStats *d = nullptr;
  unsigned long long *bc = nullptr;
  BSP_TRY(dalloc(&d, 1, s));
  BSP_TRY(dalloc(&bc, 2, s));
  BSP_CUDA(cudaMemsetAsync(d, 0, sizeof(RowStats), s));
  BSP_CUDA(cudaMemsetAsync(bc, 0, 2 * sizeof(unsigned long long), s));
  if (rows > 0) {
    row_stats_kernel<<<grid_for(rows), 256, 0, s>>>(rows, rowPtr, d);
    BSP_LAUNCH_CHECK();
    block_count_kernel<4><<<grid_for(ceil_div(rows, 4)), 256, 0, s>>>(rows, rowPtr, colIdx, bc);
    BSP_LAUNCH_CHECK();
    block_count_kernel<8><<<grid_for(ceil_div(rows, 8)), 256, 0, s>>>(rows, rowPtr, colIdx, bc + 1);
    BSP_LAUNCH_CHECK();
  }
  RowStats h{};
  unsigned long long hb[2] = {0, 0};
  BSP_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaMemcpyAsync(hb, bc, sizeof(hb), cudaMemcpyDeviceToHost, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  dfree(d, s);
  dfree(bc, s);
  const double mean = rows > 0 ? (double)nnz / rows : 0.0;
  const double var = rows > 0 ? (double)h.sum_sq / rows - mean * mean : 0.0;
  r.mean_len = mean;
  r.cv_len = mean > 0 ? std::sqrt(var > 0 ? var : 0.0) / mean : 0.0;
  r.max_len = h.max_len;
  r.long_rows = (int32_t)h.long_rows;
  r.fill4 = hb[0] ? (double)nnz / (16.0 * (double)hb[0]) : 0.0;
  r.fill8 = hb[1] ? (double)nnz / (64.0 * (double)hb[1]) : 0.0;
  return BSP_OK;
}

static void model_choice(int32_t rows, int32_t nnz, bsp_tune_result &r) {
  r.format = BSP_FMT_CSR;
  r.csr_algo = BSP_CSR_VECTOR;
  r.lanes = auto_lanes(rows, nnz);
  r.bs = 0;
  r.bsr_algo = BSP_BSR_FFMA;
  // modelled time per nonzero (bytes / relative efficiency)
  const double t_csr = 12.0 / 0.7;
  const double t_b4 = r.fill4 > 0 ? (8.0 * 16 + 4) / (16.0 * r.fill4) / 1.05 : 1e30;
  const double t_b8 = r.fill8 > 0 ? (8.0 * 64 + 4) / (64.0 * r.fill8) / 1.05 : 1e30;
  const bool skewed = r.max_len >= 256 && r.max_len > 32.0 * r.mean_len;
  if (std::min(t_b4, t_b8) < t_csr) {
    r.format = BSP_FMT_BSR;
    r.bs = t_b8 < t_b4 ? 8 : 4;
  } else if (skewed) {
    r.format = BSP_FMT_DASP;
  }
}

}  // namespace bsp

using namespace bsp;

struct bsp_spmv_plan_s {
  int32_t rows = 0, cols = 0, nnz = 0;
  const int32_t *rowPtr = nullptr, *colIdx = nullptr;
  const double *values = nullptr;
  bsp_tune_result choice{};
  bool has_bsr = false, has_dasp = false;
  bsp_bsr bsr{};
  bsp_dasp dasp{};
  void *ws = nullptr;  // merge workspace
  size_t ws_bytes = 0;
};

namespace bsp {

// Builds what `c` needs inside P (conversion or workspace).
static bsp_status materialize(bsp_spmv_plan P, const bsp_tune_result &c, cudaStream_t s) {
  if (c.format == BSP_FMT_BSR) {
    BSP_TRY(bsp_csr2bsr(P->rows, P->cols, P->nnz, P->rowPtr, P->colIdx, P->values, c.bs, &P->bsr, s));
    P->has_bsr = true;
  } else if (c.format == BSP_FMT_DASP) {
    BSP_TRY(bsp_csr2dasp(P->rows, P->cols, P->nnz, P->rowPtr, P->colIdx, P->values, 0.75, 256, &P->dasp, s));
    P->has_dasp = true;
  } else if (c.csr_algo == BSP_CSR_MERGE) {
    P->ws_bytes = bsp_csr_merge_workspace(P->rows, P->nnz);
    BSP_CUDA(cudaMallocAsync(&P->ws, P->ws_bytes ? P->ws_bytes : 16, s));
  }
  P->choice = c;
  return BSP_OK;
}

static void release(bsp_spmv_plan P) {
  if (P->has_bsr) bsp_bsr_free(&P->bsr);
  if (P->has_dasp) bsp_dasp_free(&P->dasp);
  if (P->ws) cudaFree(P->ws);
  P->has_bsr = P->has_dasp = false;
  P->ws = nullptr;
  P->ws_bytes = 0;
}

static bsp_status run(bsp_spmv_plan P, const double *x, double *y, double a, double b, cudaStream_t s) {
  const bsp_tune_result &c = P->choice;
  if (c.format == BSP_FMT_BSR) return bsp_bsr_spmv(&P->bsr, x, y, a, b, c.bsr_algo, s);
  if (c.format == BSP_FMT_DASP) return bsp_dasp_spmv(&P->dasp, x, y, a, b, 0, s);
  if (c.csr_algo == BSP_CSR_MERGE)
    return bsp_csr_spmv_merge_f64(P->rows, P->cols, P->nnz, P->rowPtr, P->colIdx, P->values, x, y, a, b, P->ws,
                                  P->ws_bytes, s);
  return bsp_csr_spmv(P->rows, P->cols, P->nnz, P->rowPtr, P->colIdx, P->values, BSP_F64, x, y, a, b,
                      BSP_CSR_VECTOR, c.lanes, s);
}

// Times `reps` runs of the current choice (after 2 warm-up runs).
static bsp_status time_choice(bsp_spmv_plan P, const double *x, double *y, int reps, double *us, cudaStream_t s) {
  cudaEvent_t e0, e1;
  BSP_CUDA(cudaEventCreate(&e0));
  BSP_CUDA(cudaEventCreate(&e1));
  bsp_status st = BSP_OK;
  for (int i = 0; i < 2 && st == BSP_OK; ++i) st = run(P, x, y, 1.0, 0.0, s);
  cudaEventRecord(e0, s);
  for (int i = 0; i < reps && st == BSP_OK; ++i) st = run(P, x, y, 1.0, 0.0, s);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *us = 1e3 * ms / reps;
  return st;
}

static bsp_status measure_choice(bsp_spmv_plan P, bsp_tune_result &r, cudaStream_t s) {
  double *x = nullptr, *y = nullptr;
  BSP_TRY(dalloc(&x, (size_t)(P->cols > 0 ? P->cols : 1), s));
  BSP_TRY(dalloc(&y, (size_t)(P->rows > 0 ? P->rows : 1), s));
  BSP_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (P->cols > 0 ? P->cols : 1), s));
  std::vector<bsp_tune_result> cand;
  for (int l = 1; l <= 32; l <<= 1) {
    bsp_tune_result c = r;
    c.format = BSP_FMT_CSR;
    c.csr_algo = BSP_CSR_VECTOR;
    c.lanes = l;
    cand.push_back(c);
  }
  {
    bsp_tune_result c = r;
    c.format = BSP_FMT_CSR;
    c.csr_algo = BSP_CSR_MERGE;
    cand.push_back(c);
  }
  if (r.max_len >= 32) {
    bsp_tune_result c = r;
    c.format = BSP_FMT_DASP;
    cand.push_back(c);
  }
  for (int bs : {4, 8}) {
    const double fill = bs == 4 ? r.fill4 : r.fill8;
    if (fill < 0.3) continue;
    bsp_tune_result c = r;
    c.format = BSP_FMT_BSR;
    c.bs = bs;
    c.bsr_algo = BSP_BSR_FFMA;
    cand.push_back(c);
  }
  bsp_status st = BSP_OK;
  double best = 1e30;
  bsp_tune_result pick = r;
  for (const auto &c : cand) {
    st = materialize(P, c, s);
    double us = 0;
    if (st == BSP_OK) st = time_choice(P, x, y, 10, &us, s);
    release(P);
    if (st != BSP_OK) break;
    if (us < best) {
      best = us;
      pick = c;
    }
  }
  dfree(x, s);
  dfree(y, s);
  BSP_CUDA(cudaStreamSynchronize(s));
  if (st != BSP_OK) return st;
  pick.spmv_us = best;
  r = pick;
  return BSP_OK;
}

static bsp_status tune_into(bsp_spmv_plan P, int32_t measure, bsp_tune_result &r, cudaStream_t s) {
  uint64_t key = 0;
  BSP_TRY(matrix_key(P->rows, P->nnz, P->rowPtr, P->colIdx, P->cols, &key, s));
  {
    std::lock_guard<std::mutex> g(g_mu);
    load_file_locked();
    auto it = g_cache.find(key);
    // a cached model choice does not answer a measure request
    if (it != g_cache.end() && (!measure || it->second.spmv_us > 0)) {
      r = it->second;
      r.from_cache = 1;
      return BSP_OK;
    }
  }
  r = bsp_tune_result{};
  r.key = key;
  BSP_TRY(stats(P->rows, P->nnz, P->rowPtr, P->colIdx, r, s));
  model_choice(P->rows, P->nnz, r);
  if (measure) BSP_TRY(measure_choice(P, r, s));
  r.from_cache = 0;
  std::lock_guard<std::mutex> g(g_mu);
  g_cache[key] = r;
  append_file_locked(r);
  return BSP_OK;
}

}  // namespace bsp

extern "C" bsp_status bsp_matrix_key(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                     const int32_t *colIdx, uint64_t *key, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(key && rowPtr && rows >= 0 && nnz >= 0 && (nnz == 0 || colIdx), "bad argument");
  return matrix_key(rows, nnz, rowPtr, colIdx, cols, key, as_stream(stream));
}

extern "C" void bsp_tune_cache_clear(void) {
  std::lock_guard<std::mutex> g(g_mu);
  g_cache.clear();
}

extern "C" bsp_status bsp_spmv_plan_create(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                           const int32_t *colIdx, const double *values, int32_t measure,
                                           bsp_spmv_plan *plan, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(plan && rowPtr && rows >= 0 && cols >= 0 && nnz >= 0, "bad argument");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values), "null pointer");
  *plan = nullptr;
  cudaStream_t s = as_stream(stream);
  bsp_spmv_plan P = new bsp_spmv_plan_s();
  P->rows = rows;
  P->cols = cols;
  P->nnz = nnz;
  P->rowPtr = rowPtr;
  P->colIdx = colIdx;
  P->values = values;
  bsp_tune_result r{};
  bsp_status st = tune_into(P, measure, r, s);
  if (st == BSP_OK) st = materialize(P, r, s);
  if (st == BSP_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? BSP_OK : BSP_ERR_CUDA;
  if (st != BSP_OK) {
    release(P);
    delete P;
    return st;
  }
  *plan = P;
  return BSP_OK;
}

extern "C" bsp_status bsp_tune_spmv(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                    const int32_t *colIdx, const double *values, int32_t measure,
                                    bsp_tune_result *out, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(out && rowPtr && rows >= 0 && cols >= 0 && nnz >= 0, "bad argument");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values), "null pointer");
  bsp_spmv_plan_s P;
  P.rows = rows;
  P.cols = cols;
  P.nnz = nnz;
  P.rowPtr = rowPtr;
  P.colIdx = colIdx;
  P.values = values;
  const bsp_status st = tune_into(&P, measure, *out, as_stream(stream));
  release(&P);
  return st;
}

extern "C" bsp_status bsp_spmv_plan_choice(bsp_spmv_plan plan, bsp_tune_result *out) {
  clear_error();
  BSP_CHECK_ARG(plan && out, "null pointer");
  *out = plan->choice;
  return BSP_OK;
}

extern "C" bsp_status bsp_spmv_plan_run(bsp_spmv_plan plan, const double *x, double *y, double alpha,
                                        double beta, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(plan && (plan->cols == 0 || x) && (plan->rows == 0 || y), "null pointer");
  if (plan->rows == 0) return BSP_OK;
  return run(plan, x, y, alpha, beta, as_stream(stream));
}

extern "C" bsp_status bsp_spmv_plan_destroy(bsp_spmv_plan plan) {
  clear_error();
  if (!plan) return BSP_OK;
  release(plan);
  cudaDeviceSynchronize();
  delete plan;
  return BSP_OK;
}
