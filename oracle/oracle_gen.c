/*
 * oracle_gen.c — input generator for the CPU side of the benchmark.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  The reference arm of bench.py
 * times the reference's CPU SpMV (src/ref.cpp:26-37) on the headline matrix;
 * it builds that matrix here, so the process that times the reference never
 * loads the library under test.
 *
 * The matrix and vector are the seeded synthetic inputs of the benchmark: a
 * 27-point stencil on an m^3 grid with `dof` unknowns per node (every node
 * couples all dof unknowns of each of its up-to-27 neighbours, block fill
 * 100%), values N(0,1) by Box-Muller from a counter-based splitmix64 hash of
 * (seed, stream, index), and x uniform in [-1, 1) from the same hash.  Each
 * draw depends only on its index, so the result is independent of the thread
 * count.  tests/test_generators.py checks this file bit for bit against the
 * library's generator.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "oracle.h"

static uint64_t gen_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t gen_hash(uint64_t seed, uint64_t stream, uint64_t idx) {
  return gen_mix64(gen_mix64(gen_mix64(seed) ^ stream) ^ (idx * 0xD6E8FEB86659FD93ull));
}

/* Uniform in (0, 1) from the top 53 bits, never 0. */
static double gen_open01(uint64_t h) { return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

enum { STREAM_VAL = 1, STREAM_X = 6 };

static double gen_normal(uint64_t seed, uint64_t idx) {
  const double u1 = gen_open01(gen_hash(seed, STREAM_VAL, 2 * idx));
  const double u2 = gen_open01(gen_hash(seed, STREAM_VAL, 2 * idx + 1));
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static int gen_span(int64_t c, int64_t m) { return 1 + (c > 0) + (c < m - 1); }

int64_t orc_gen_stencil27(int32_t m, int32_t dof, uint64_t seed, int32_t *rowPtr, int32_t *colIdx, double *val) {
  if (m <= 0 || dof <= 0) return -1;
  const int64_t nodes = (int64_t)m * m * m, n = nodes * dof;
  if (n > INT32_MAX) return -1;
  /* row pointers: a node's rows each hold (neighbour count) * dof entries */
  int64_t acc = 0;
  for (int64_t node = 0; node < nodes; ++node) {
    const int64_t x = node % m, y = (node / m) % m, z = node / ((int64_t)m * m);
    const int64_t len = (int64_t)gen_span(x, m) * gen_span(y, m) * gen_span(z, m) * dof;
    for (int d = 0; d < dof; ++d) {
      if (rowPtr) rowPtr[node * dof + d] = (int32_t)acc;
      acc += len;
    }
  }
  if (rowPtr) rowPtr[n] = (int32_t)acc;
  if (acc > INT32_MAX) return -1;
  if (!rowPtr || !colIdx || !val) return acc;
#pragma omp parallel for schedule(static)
  for (int64_t row = 0; row < n; ++row) {
    const int64_t node = row / dof;
    const int64_t x = node % m, y = (node / m) % m, z = node / ((int64_t)m * m);
    int64_t k = rowPtr[row];
    for (int64_t zz = z - 1; zz <= z + 1; ++zz)
      for (int64_t yy = y - 1; yy <= y + 1; ++yy)
        for (int64_t xx = x - 1; xx <= x + 1; ++xx) {
          if (xx < 0 || yy < 0 || zz < 0 || xx >= m || yy >= m || zz >= m) continue;
          const int64_t base = ((zz * m + yy) * m + xx) * dof;
          for (int e = 0; e < dof; ++e, ++k) {
            colIdx[k] = (int32_t)(base + e);
            val[k] = gen_normal(seed, (uint64_t)k);
          }
        }
  }
  return acc;
}

void orc_gen_uniform(int64_t n, uint64_t seed, double *x) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = 2.0 * gen_open01(gen_hash(seed, STREAM_X, (uint64_t)i)) - 1.0;
}
