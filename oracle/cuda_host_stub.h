// Shared declarations of the CPU CUDA-runtime stub (cuda_host_stub.cpp).
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <stddef.h>
#include <vector>

struct StubAlloc {
  void *ptr;
  size_t bytes;
  size_t uploaded;
};
struct StubLaunch {
  const void *func;
  unsigned grid[3], block[3];
  void **args;  // valid only inside stub_on_launch
  int nargs;
};
extern std::vector<StubAlloc> g_allocs;
extern std::vector<StubLaunch> g_launches;
// Index of the stub allocation containing p (and the byte offset), or -1.
int stub_alloc_index(const void *p, size_t *offset);
// Called synchronously for every kernel launch (defined by the capture main).
void stub_on_launch(const StubLaunch &L);
