// CPU stand-in for the 13 CUDA runtime entry points that the reference's
// src/dasp.cu host code calls (cudaMalloc/Memcpy/Memset/Free/
// DeviceSynchronize/FuncSetAttribute/LaunchKernel and the fat-binary
// registration hooks nvcc emits).  TEST INFRASTRUCTURE ONLY: linked into
// oracle/_ref/dasp_capture so that the reference's own packing code
// (spmv_all, dasp.cu:814-1600) runs on the CPU and every array it uploads
// to the "device", plus every kernel launch with its arguments, can be
// recorded and compared with the library's device-side packing.
//
// "Device" allocations are host allocations; nothing is freed until the
// capture is written, so uploaded contents survive spmv_all's cudaFree.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "cuda_host_stub.h"

namespace {
struct Dim3 {
  unsigned x, y, z;
};
}  // namespace

std::vector<StubAlloc> g_allocs;
std::vector<StubLaunch> g_launches;
static Dim3 g_cfg_grid, g_cfg_block;
static size_t g_cfg_shmem;
static void *g_cfg_stream;

int stub_alloc_index(const void *p, size_t *offset) {
  for (size_t i = 0; i < g_allocs.size(); ++i) {
    const char *b = (const char *)g_allocs[i].ptr;
    if ((const char *)p >= b && (const char *)p < b + (g_allocs[i].bytes ? g_allocs[i].bytes : 1)) {
      if (offset) *offset = (const char *)p - b;
      return (int)i;
    }
  }
  return -1;
}

extern "C" {

void **__cudaRegisterFatBinary(void *) {
  static void *handle = nullptr;
  return &handle;
}
void __cudaRegisterFatBinaryEnd(void **) {}
void __cudaUnregisterFatBinary(void **) {}
void __cudaRegisterFunction(void **, const char *, char *, const char *, int, void *, void *, void *, void *,
                            int *) {}

unsigned __cudaPushCallConfiguration(Dim3 grid, Dim3 block, size_t shmem, void *stream) {
  g_cfg_grid = grid;
  g_cfg_block = block;
  g_cfg_shmem = shmem;
  g_cfg_stream = stream;
  return 0;
}
int __cudaPopCallConfiguration(Dim3 *grid, Dim3 *block, size_t *shmem, void *stream) {
  *grid = g_cfg_grid;
  *block = g_cfg_block;
  *shmem = g_cfg_shmem;
  if (stream) *(void **)stream = g_cfg_stream;
  return 0;
}

// Records the launch; the argument vector is copied as raw 8-byte slots
// (every dasp_spmv2 / longPart_sum parameter is a pointer or a 4-byte int).
int cudaLaunchKernel(const void *func, Dim3 grid, Dim3 block, void **args, size_t, void *) {
  StubLaunch L;
  L.func = func;
  L.grid[0] = grid.x;
  L.grid[1] = grid.y;
  L.grid[2] = grid.z;
  L.block[0] = block.x;
  L.block[1] = block.y;
  L.block[2] = block.z;
  L.args = args;  // resolved by the caller of spmv_all through stub_decode_args
  L.nargs = 0;
  g_launches.push_back(L);
  stub_on_launch(g_launches.back());
  return 0;
}

int cudaMalloc(void **p, size_t bytes) {
  void *q = calloc(bytes ? bytes : 1, 1);
  if (!q) return 2;
  g_allocs.push_back(StubAlloc{q, bytes, 0});
  *p = q;
  return 0;
}
int cudaMemcpy(void *dst, const void *src, size_t bytes, int kind) {
  (void)kind;
  if (bytes) memcpy(dst, src, bytes);
  size_t off = 0;
  const int i = stub_alloc_index(dst, &off);
  if (i >= 0) g_allocs[i].uploaded += bytes;
  return 0;
}
int cudaMemset(void *p, int v, size_t bytes) {
  if (bytes) memset(p, v, bytes);
  return 0;
}
int cudaFree(void *) { return 0; }
int cudaDeviceSynchronize(void) { return 0; }
int cudaFuncSetAttribute(const void *, int, int) { return 0; }

}  // extern "C"
