// Host-buffer BSR SpMV with the transfers overlapped (no reference
// counterpart; the reference's amgT_spmv_fp64, src/amgT.cu:1355, copies x,
// runs, and copies y back one after the other).
//
// The block rows are cut into `chunks` ranges.  x goes up in as many
// equal pieces on one stream, each recording an event; block-row range c
// waits only for the x pieces up to the one holding its largest column
// (computed once at plan time), runs on a second stream, and its y piece
// goes down on a third stream as soon as it is done.  For matrices whose
// columns follow their rows (stencils, banded, reordered matrices) the
// upload, the SpMV and the download overlap; with pinned host buffers the
// two copy directions also run at the same time.
#include <algorithm>
#include <vector>

#include "bsp_internal.cuh"
#include "util.cuh"

namespace bsp {

bsp_status bsr_spmv_rows(const bsp_bsr *m, int32_t lo, int32_t hi, const double *x, double *y, double alpha,
                         double beta, int64_t max_blocks, cudaStream_t s);

// Largest block column of each block-row range (atomicMax per range).
__global__ void chunk_maxcol_kernel(int32_t nchunks, const int32_t *__restrict__ lo,
                                    const int32_t *__restrict__ blcPtr, const int32_t *__restrict__ blcIdx,
                                    int32_t *__restrict__ maxcol) {
  for (int32_t c = blockIdx.y; c < nchunks; c += gridDim.y) {
    const int32_t b0 = blcPtr[lo[c]], b1 = blcPtr[lo[c + 1]];
    int32_t m = -1;
    for (int64_t k = b0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < b1;
         k += (int64_t)gridDim.x * blockDim.x)
      m = max(m, blcIdx[k]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m >= 0) atomicMax(&maxcol[c], m);
  }
}

}  // namespace bsp

using namespace bsp;

struct bsp_bsr_host_plan_s {
  const bsp_bsr *m = nullptr;
  int32_t chunks = 0;
  std::vector<int32_t> lo;        // [chunks+1] block-row ranges
  std::vector<int32_t> need;      // [chunks] last x piece each range reads
  std::vector<int64_t> xoff;      // [chunks+1] x pieces (elements)
  double *dx = nullptr, *dy = nullptr;
  cudaStream_t up = nullptr, run = nullptr, down = nullptr;
  std::vector<cudaEvent_t> xev, yev;
  cudaEvent_t start = nullptr;
  // the whole fork/join sequence as a CUDA graph, kept for the last
  // (x_host, y_host, alpha, beta): one launch per call when they repeat
  cudaStream_t origin = nullptr;
  cudaGraphExec_t graph = nullptr;
  const double *g_x = nullptr;
  double *g_y = nullptr;
  double g_alpha = 0.0, g_beta = 0.0;
  int32_t use_graph = 1;
  // grid cap of each range's SpMV (0 = the kernel's own grid).  Default: one
  // wave, 8 CTAs of 256 per SM, the rows walked by grid stride (27-point
  // stencil 64^3 x 4 dof, 8 ranges, pinned 8 MB up and down per call: 311-316
  // us per call against 316-327 us with the kernel's 1.7-wave grid, four
  // interleaved repetitions; 6 CTAs per SM 334-338 us)
  int32_t max_ctas = 0;
};

static void plan_release(bsp_bsr_host_plan_s *P) {
  if (P->graph) cudaGraphExecDestroy(P->graph);
  if (P->origin) cudaStreamDestroy(P->origin);
  for (cudaEvent_t e : P->xev) cudaEventDestroy(e);
  for (cudaEvent_t e : P->yev) cudaEventDestroy(e);
  if (P->start) cudaEventDestroy(P->start);
  if (P->up) cudaStreamDestroy(P->up);
  if (P->run) cudaStreamDestroy(P->run);
  if (P->down) cudaStreamDestroy(P->down);
  if (P->dx) cudaFree(P->dx);
  if (P->dy) cudaFree(P->dy);
  delete P;
}

extern "C" bsp_status bsp_bsr_host_plan_create(const bsp_bsr *m, int32_t chunks, bsp_bsr_host_plan *out,
                                               bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(m && out, "null pointer");
  BSP_CHECK_ARG(m->bs == 4 || m->bs == 8, "block size must be 4 or 8");
  BSP_CHECK_ARG(chunks >= 1 && chunks <= 64, "chunks must be in [1, 64]");
  *out = nullptr;
  cudaStream_t s = as_stream(stream);
  auto *P = new bsp_bsr_host_plan_s();
  P->m = m;
  P->max_ctas = sm_count() * 8;
  P->chunks = std::max<int32_t>(1, std::min<int32_t>(chunks, std::max<int32_t>(1, m->blc_row)));
  const int32_t C = P->chunks;
  P->lo.resize(C + 1);
  for (int32_t c = 0; c <= C; ++c) P->lo[c] = (int32_t)((int64_t)m->blc_row * c / C);
  P->xoff.resize(C + 1);
  for (int32_t c = 0; c <= C; ++c) P->xoff[c] = (int64_t)m->col * c / C;
  auto fail = [&](bsp_status st, const char *msg) {
    plan_release(P);
    BSP_FAIL(st, msg);
  };
  // largest block column per range -> last x piece it needs
  int32_t *dlo = nullptr, *dmax = nullptr;
  if (dalloc(&dlo, (size_t)C + 1, s) != BSP_OK || dalloc(&dmax, (size_t)C, s) != BSP_OK)
    return fail(BSP_ERR_ALLOC, "allocating the plan's scratch failed");
  cudaMemcpyAsync(dlo, P->lo.data(), sizeof(int32_t) * (C + 1), cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(dmax, 0xff, sizeof(int32_t) * C, s);  // -1
  if (m->blc_row > 0) {
    chunk_maxcol_kernel<<<dim3(64, (unsigned)C), 256, 0, s>>>(C, dlo, m->blcPtr, m->blcIdx, dmax);
  }
  std::vector<int32_t> maxcol(C);
  cudaMemcpyAsync(maxcol.data(), dmax, sizeof(int32_t) * C, cudaMemcpyDeviceToHost, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  dfree(dlo, s);
  dfree(dmax, s);
  if (e != cudaSuccess) return fail(BSP_ERR_CUDA, cudaGetErrorString(e));
  P->need.resize(C);
  for (int32_t c = 0; c < C; ++c) {
    const int64_t last_col = maxcol[c] < 0 ? 0 : std::min<int64_t>((int64_t)maxcol[c] * m->bs + m->bs - 1,
                                                                   (int64_t)m->col - 1);
    int32_t j = 0;
    while (j + 1 < C && P->xoff[j + 1] <= last_col) ++j;
    P->need[c] = j;
  }
  if (cudaMalloc(&P->dx, sizeof(double) * std::max<int64_t>(1, m->col)) != cudaSuccess ||
      cudaMalloc(&P->dy, sizeof(double) * std::max<int64_t>(1, m->row)) != cudaSuccess)
    return fail(BSP_ERR_ALLOC, "allocating x / y failed");
  if (cudaStreamCreateWithFlags(&P->up, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&P->run, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&P->down, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&P->origin, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&P->start, cudaEventDisableTiming) != cudaSuccess)
    return fail(BSP_ERR_CUDA, "creating streams failed");
  P->xev.resize(C, nullptr);
  P->yev.resize(C, nullptr);
  for (int32_t c = 0; c < C; ++c)
    if (cudaEventCreateWithFlags(&P->xev[c], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&P->yev[c], cudaEventDisableTiming) != cudaSuccess)
      return fail(BSP_ERR_CUDA, "creating events failed");
  *out = P;
  return BSP_OK;
}

// Enqueues the pipeline after `s` and joins it back into `s`.
static bsp_status enqueue(bsp_bsr_host_plan P, const double *x_host, double *y_host, double alpha, double beta,
                          cudaStream_t s) {
  const bsp_bsr *m = P->m;
  const int32_t C = P->chunks, bs = m->bs;
  BSP_CUDA(cudaEventRecord(P->start, s));
  BSP_CUDA(cudaStreamWaitEvent(P->up, P->start, 0));
  BSP_CUDA(cudaStreamWaitEvent(P->run, P->start, 0));
  BSP_CUDA(cudaStreamWaitEvent(P->down, P->start, 0));
  for (int32_t j = 0; j < C; ++j) {
    const int64_t a = P->xoff[j], b = P->xoff[j + 1];
    if (b > a)
      BSP_CUDA(cudaMemcpyAsync(P->dx + a, x_host + a, sizeof(double) * (b - a), cudaMemcpyHostToDevice, P->up));
    BSP_CUDA(cudaEventRecord(P->xev[j], P->up));
  }
  for (int32_t c = 0; c < C; ++c) {
    const int64_t r0 = (int64_t)P->lo[c] * bs, r1 = std::min<int64_t>((int64_t)P->lo[c + 1] * bs, m->row);
    BSP_CUDA(cudaStreamWaitEvent(P->run, P->xev[P->need[c]], 0));
    if (beta != 0.0 && r1 > r0)
      BSP_CUDA(cudaMemcpyAsync(P->dy + r0, y_host + r0, sizeof(double) * (r1 - r0), cudaMemcpyHostToDevice,
                               P->run));
    BSP_TRY(bsr_spmv_rows(m, P->lo[c], P->lo[c + 1], P->dx, P->dy, alpha, beta, P->max_ctas, P->run));
    BSP_CUDA(cudaEventRecord(P->yev[c], P->run));
    BSP_CUDA(cudaStreamWaitEvent(P->down, P->yev[c], 0));
    if (r1 > r0)
      BSP_CUDA(cudaMemcpyAsync(y_host + r0, P->dy + r0, sizeof(double) * (r1 - r0), cudaMemcpyDeviceToHost,
                               P->down));
  }
  // join: `s` continues after the last download and the x upload
  BSP_CUDA(cudaEventRecord(P->xev[C - 1], P->up));
  BSP_CUDA(cudaStreamWaitEvent(s, P->xev[C - 1], 0));
  BSP_CUDA(cudaEventRecord(P->yev[C - 1], P->down));
  BSP_CUDA(cudaStreamWaitEvent(s, P->yev[C - 1], 0));
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_spmv_host_pipelined(bsp_bsr_host_plan P, const double *x_host, double *y_host,
                                                  double alpha, double beta, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(P && x_host && y_host, "null pointer");
  cudaStream_t s = as_stream(stream);
  if (!P->use_graph) {
    BSP_TRY(enqueue(P, x_host, y_host, alpha, beta, s));
    BSP_CUDA(cudaStreamSynchronize(s));
    return BSP_OK;
  }
  const bool same = P->graph && P->g_x == x_host && P->g_y == y_host && P->g_alpha == alpha && P->g_beta == beta;
  if (!same) {
    if (P->graph) {
      cudaGraphExecDestroy(P->graph);
      P->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    BSP_CUDA(cudaStreamBeginCapture(P->origin, cudaStreamCaptureModeThreadLocal));
    const bsp_status st = enqueue(P, x_host, y_host, alpha, beta, P->origin);
    const cudaError_t e = cudaStreamEndCapture(P->origin, &g);
    if (st != BSP_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    BSP_CUDA(e);
    const cudaError_t ei = cudaGraphInstantiate(&P->graph, g, 0);
    cudaGraphDestroy(g);
    BSP_CUDA(ei);
    P->g_x = x_host;
    P->g_y = y_host;
    P->g_alpha = alpha;
    P->g_beta = beta;
  }
  BSP_CUDA(cudaGraphLaunch(P->graph, s));
  BSP_CUDA(cudaStreamSynchronize(s));
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_host_plan_set_graph(bsp_bsr_host_plan P, int32_t use_graph) {
  clear_error();
  BSP_CHECK_ARG(P, "null plan");
  P->use_graph = use_graph ? 1 : 0;
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_host_plan_set_ctas(bsp_bsr_host_plan P, int32_t max_ctas) {
  clear_error();
  BSP_CHECK_ARG(P, "null plan");
  BSP_CHECK_ARG(max_ctas >= 0, "max_ctas must be >= 0");
  if (P->max_ctas != max_ctas && P->graph) {   // the recorded graph holds the old grids
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  P->max_ctas = max_ctas;
  return BSP_OK;
}

extern "C" bsp_status bsp_bsr_host_plan_destroy(bsp_bsr_host_plan P) {
  clear_error();
  if (!P) return BSP_OK;
  cudaStreamSynchronize(P->up);
  cudaStreamSynchronize(P->run);
  cudaStreamSynchronize(P->down);
  plan_release(P);
  return BSP_OK;
}
