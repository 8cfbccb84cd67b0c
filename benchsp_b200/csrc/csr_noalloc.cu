// Allocation-free variant of the FP64 merge-path CSR SpMV.
//
// The regular merge-path entry points either allocate their carry workspace
// (bsp_csr_spmv with BSP_CSR_MERGE) or take one from the caller
// (bsp_csr_spmv_merge_f64).  Some hosts can do neither: a serving process
// that hands all device memory to its own pool at start-up and forbids any
// further cudaMalloc, or a latency-critical loop where cudaMalloc/cudaFree
// (which can synchronize the device) must not appear after initialization.
// For them this file keeps the workspace in a fixed device array that is
// part of the library image, so a call needs no allocation at all.
//
// The array is a file-scope __device__ variable.  Host code may not use its
// name as a pointer (on the host the name is only a stand-in for the
// symbol), so the device address is looked up with cudaGetSymbolAddress
// once per device, on that device's first call, and cached.
#include <mutex>

#include "bsp_internal.cuh"

namespace bsp {

bsp_status launch_merge(int32_t rows, int32_t nnz, const int32_t *rowPtr, const int32_t *colIdx,
                        const double *val, const double *x, double *y, double alpha, double beta,
                        int32_t *carry_row, double *carry_val, cudaStream_t s);

// One carry slot (int32 row + FP64 partial) per merge-path warp of 256 merge
// items; rows + nnz is limited to 262,144 warps * 256 = 67,108,864 items,
// which fixes the array at 3 MiB per device.
constexpr int64_t kNoAllocMaxWarps = 262144;
constexpr int64_t kNoAllocMaxItems = kNoAllocMaxWarps * 256;
constexpr size_t kNoAllocRowBytes = (size_t)kNoAllocMaxWarps * sizeof(int32_t);
constexpr size_t kNoAllocBytes = kNoAllocRowBytes + (size_t)kNoAllocMaxWarps * sizeof(double);
static_assert(kNoAllocRowBytes % 256 == 0, "carry values must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_merge_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[kNoAllocMaxDevices];

// Device address of the array on the current device (looked up on first use).
static bsp_status noalloc_scratch(void **out) {
  int dev = 0;
  BSP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) BSP_FAIL(BSP_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    BSP_CUDA(cudaGetSymbolAddress(&p, g_merge_noalloc_scratch));
    if (!p) BSP_FAIL(BSP_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return BSP_OK;
}

}  // namespace bsp

using namespace bsp;

extern "C" bsp_status bsp_csr_spmv_merge_f64_noalloc(int32_t rows, int32_t cols, int32_t nnz,
                                                     const int32_t *rowPtr, const int32_t *colIdx,
                                                     const double *values, const double *x, double *y,
                                                     double alpha, double beta, bsp_stream_t stream) {
  clear_error();
  BSP_CHECK_ARG(rows >= 0 && cols >= 0 && nnz >= 0, "negative size");
  if ((int64_t)rows + nnz > kNoAllocMaxItems)
    BSP_FAIL(BSP_ERR_INVALID, "rows + nnz = " + std::to_string((int64_t)rows + nnz) +
                                  " exceeds the allocation-free limit of 67108864 (use bsp_csr_spmv_merge_f64)");
  if (rows == 0) return BSP_OK;
  BSP_CHECK_ARG(rowPtr && y, "null pointer");
  BSP_CHECK_ARG(nnz == 0 || (colIdx && values && x), "null pointer");
  void *scratch = nullptr;
  BSP_TRY(noalloc_scratch(&scratch));
  // Every carry slot the fix-up reads is written by the main kernel of the
  // same call, so nothing has to be cleared between calls.
  int32_t *carry_row = reinterpret_cast<int32_t *>(scratch);
  double *carry_val = reinterpret_cast<double *>(reinterpret_cast<char *>(scratch) + kNoAllocRowBytes);
  return launch_merge(rows, nnz, rowPtr, colIdx, values, x, y, alpha, beta, carry_row, carry_val,
                      as_stream(stream));
}
