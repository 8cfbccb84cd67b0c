/*
 * oracle.c — CPU restatement of the reference's hot-path algorithms.
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the parity tests,
 * never part of the library.  Compiled with -ffp-contract=off so every
 * multiply and add is rounded separately, as the reference's x86 build of
 * src/ref.cpp does.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_spmv_f64(int64_t rows, const int64_t *rowPtr, const int64_t *colIdx, const double *val,
                  const double *x, double *y) {
  /* src/ref.cpp:26-37 */
  for (int64_t i = 0; i < rows; i++) {
    double sum = 0;
    for (int64_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) sum += val[j] * x[colIdx[j]];
    y[i] = sum;
  }
}

void orc_spmv_f64_i32(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                      const double *x, double *y) {
  for (int32_t i = 0; i < rows; i++) {
    double sum = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) sum += val[j] * x[colIdx[j]];
    y[i] = sum;
  }
}

void orc_spmv_f32(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const float *val,
                  const float *x, float *y) {
  /* src/ref.cpp:14-24 */
  for (int32_t i = 0; i < rows; i++) {
    float sum = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) sum += val[j] * x[colIdx[j]];
    y[i] = sum;
  }
}

/* IEEE binary16 <-> binary32 by bit manipulation (round to nearest even). */
uint16_t orc_f32_to_f16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  const uint32_t sign = (u >> 16) & 0x8000u;
  const uint32_t absu = u & 0x7fffffffu;
  if (absu >= 0x7f800000u) /* inf or nan */
    return (uint16_t)(sign | 0x7c00u | (absu > 0x7f800000u ? 0x200u : 0u));
  if (absu >= 0x477ff000u) /* rounds to >= 65520 -> inf */
    return (uint16_t)(sign | 0x7c00u);
  if (absu < 0x38800000u) { /* result is a half subnormal (or zero) */
    if (absu < 0x33000000u) return (uint16_t)sign; /* <= 2^-25 rounds to 0 */
    const uint32_t e = absu >> 23;
    const uint32_t mant = (absu & 0x7fffffu) | 0x800000u;
    /* value = mant * 2^(e-150); in units of 2^-24 drop (126 - e) bits */
    const uint32_t sh = 126 - e;
    uint32_t q = mant >> sh;
    const uint32_t rem = mant & ((1u << sh) - 1);
    const uint32_t halfway = 1u << (sh - 1);
    if (rem > halfway || (rem == halfway && (q & 1))) q++;
    return (uint16_t)(sign | q);
  }
  /* normal */
  uint32_t h = ((absu >> 13) - ((127 - 15) << 10));
  const uint32_t rem = absu & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1))) h++;
  return (uint16_t)(sign | h);
}

float orc_f16_to_f32(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1f, m = h & 0x3ffu;
  uint32_t u;
  if (e == 0) {
    if (m == 0) {
      u = sign;
    } else { /* subnormal: normalise */
      int k = -1;
      do {
        k++;
        m <<= 1;
      } while (!(m & 0x400u));
      u = sign | ((uint32_t)(127 - 15 - k) << 23) | ((m & 0x3ffu) << 13);
    }
  } else if (e == 31) {
    u = sign | 0x7f800000u | (m << 13);
  } else {
    u = sign | ((e + 127 - 15) << 23) | (m << 13);
  }
  float f;
  memcpy(&f, &u, 4);
  return f;
}

uint16_t orc_f32_to_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}

float orc_bf16_to_f32(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

void orc_spmv_f16(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const uint16_t *val,
                  const uint16_t *x, uint16_t *y) {
  /* src/ref.cpp:3-13: float sum of half-valued products, half result */
  for (int32_t i = 0; i < rows; i++) {
    float sum = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) sum += orc_f16_to_f32(val[j]) * orc_f16_to_f32(x[colIdx[j]]);
    y[i] = orc_f32_to_f16(sum);
  }
}

void orc_abs_rowsum(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                    const double *x, double *out) {
  for (int32_t i = 0; i < rows; i++) {
    double s = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) s += fabs(val[j] * x[colIdx[j]]);
    out[i] = s;
  }
}

/* Dense-output SpMM in FP64: C[i,:] = sum_j a_ij * B[j,:] and, for the error
 * bound, absC[i,:] = sum_j |a_ij * B[j,:]|.  The reference's SpMM
 * (src/smat.cu:22-101, FP16 accumulation) computes the same product; its
 * kernel never stores the result, so this is the mathematical oracle. */
void orc_spmm_f64(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t N,
                  const double *B, double *Cout, double *absC) {
  for (int32_t i = 0; i < rows; i++) {
    double *c = Cout + (int64_t)i * N, *a = absC + (int64_t)i * N;
    for (int32_t k = 0; k < N; k++) c[k] = a[k] = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++) {
      const double v = val[j];
      const double *b = B + (int64_t)colIdx[j] * N;
      for (int32_t k = 0; k < N; k++) {
        c[k] += v * b[k];
        a[k] += fabs(v * b[k]);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
static int cmp_i32(const void *a, const void *b) {
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

int64_t orc_csr2bsr(int32_t rows, int32_t cols, const int32_t *rowPtr, const int32_t *colIdx,
                    const double *val, int32_t bs, int32_t *blcPtr, int32_t *blcIdx, double *blcVal,
                    uint64_t *blcMap) {
  (void)cols;
  const int32_t brow = (rows + bs - 1) / bs;
  int64_t total = 0;
  int32_t cap = 64;
  int32_t *keys = (int32_t *)malloc(sizeof(int32_t) * cap);
  for (int32_t br = 0; br < brow; br++) {
    const int32_t r0 = br * bs, r1 = r0 + bs < rows ? r0 + bs : rows;
    const int32_t len = rowPtr[r1] - rowPtr[r0];
    if (len > cap) {
      cap = len;
      keys = (int32_t *)realloc(keys, sizeof(int32_t) * cap);
    }
    /* distinct block columns of the block-row, ascending: the reference
     * ranks hash entries by counting smaller keys (amgT.cu:823-835) */
    for (int32_t j = rowPtr[r0]; j < rowPtr[r1]; j++) keys[j - rowPtr[r0]] = colIdx[j] / bs;
    qsort(keys, (size_t)len, sizeof(int32_t), cmp_i32);
    int32_t nb = 0;
    for (int32_t k = 0; k < len; k++)
      if (k == 0 || keys[k] != keys[k - 1]) keys[nb++] = keys[k];
    if (blcPtr) {
      blcPtr[br] = (int32_t)total;
      for (int32_t k = 0; k < nb; k++) {
        blcIdx[total + k] = keys[k];
        blcMap[total + k] = 0;
        for (int32_t e = 0; e < bs * bs; e++) blcVal[(total + k) * bs * bs + e] = 0.0;
      }
      for (int32_t r = r0; r < r1; r++)
        for (int32_t j = rowPtr[r]; j < rowPtr[r + 1]; j++) {
          const int32_t b = colIdx[j] / bs;
          /* binary search of the block's rank (BinarySearch2, amgT.cu:36-51) */
          int32_t lo = 0, hi = nb - 1, pos = -1;
          while (lo <= hi) {
            const int32_t mid = (lo + hi) / 2;
            if (b < keys[mid])
              hi = mid - 1;
            else if (b > keys[mid])
              lo = mid + 1;
            else {
              pos = mid;
              break;
            }
          }
          const int64_t blk = total + pos;
          const int32_t ir = r - r0, ic = colIdx[j] % bs;
          blcVal[blk * bs * bs + ir * bs + ic] = val[j];
          blcMap[blk] |= 1ull << (ir * bs + ic);
        }
    }
    total += nb;
  }
  if (blcPtr) blcPtr[brow] = (int32_t)total;
  free(keys);
  return total;
}

int32_t orc_bsr_chunks(int32_t blc_row, const int32_t *blcPtr, int32_t *rowPtrbyWarp, int32_t *rowIdxbyWarp) {
  int32_t acc = 0;
  for (int32_t br = 0; br < blc_row; br++) {
    const int32_t len = blcPtr[br + 1] - blcPtr[br];
    const int32_t c = (len + 64 - 1) / 64; /* WARP_CAPACITY 64, include/common.h:7 */
    if (rowPtrbyWarp) rowPtrbyWarp[br] = acc;
    if (rowIdxbyWarp)
      for (int32_t k = 0; k < c; k++) rowIdxbyWarp[acc + k] = br;
    acc += c;
  }
  if (rowPtrbyWarp) rowPtrbyWarp[blc_row] = acc;
  return acc;
}

double orc_bsr_stand(int32_t blc_row, const int32_t *blcPtr) {
  if (blc_row <= 0) return 0.0;
  const double avg = (double)blcPtr[blc_row] / (double)blc_row;
  double s = 0.0;
  for (int32_t br = 0; br < blc_row; br++) {
    const double d = (double)(blcPtr[br + 1] - blcPtr[br]) - avg;
    s += d * d;
  }
  return (double)sqrtf((float)(s / blc_row));
}

/* FP64 CG on the CPU with orc_spmv_f64_i32 as the operator (the reference has
 * no solver; this is the FP64 oracle the GPU solves are compared against).
 * Returns iterations; x holds the solution. */
/* Inverse of the diagonal blocks of bs consecutive rows (bs = 1: the inverse
 * diagonal), row-major bs*bs per block, the last block padded with identity
 * rows; Gauss-Jordan elimination with partial pivoting.  Returns 0, or -1 on
 * a zero pivot.  No reference counterpart (the reference has no solver);
 * plain FP64 restatement of block-Jacobi preconditioning. */
int32_t orc_block_jacobi(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t bs,
                         double *minv) {
  const int64_t nb = ((int64_t)n + bs - 1) / bs;
  double *M = (double *)malloc(sizeof(double) * bs * bs * 2);
  double *I = M + bs * bs;
  int32_t rc = 0;
  for (int64_t b = 0; b < nb && rc == 0; b++) {
    const int64_t lo = b * bs;
    for (int32_t i = 0; i < bs * bs; i++) {
      M[i] = 0.0;
      I[i] = (i / bs == i % bs) ? 1.0 : 0.0;
    }
    for (int32_t i = 0; i < bs; i++) {
      if (lo + i >= n) {
        M[i * bs + i] = 1.0;
        continue;
      }
      for (int32_t j = rowPtr[lo + i]; j < rowPtr[lo + i + 1]; j++)
        if (colIdx[j] >= lo && colIdx[j] < lo + bs) M[i * bs + (colIdx[j] - lo)] += val[j];
    }
    for (int32_t c = 0; c < bs; c++) {
      int32_t piv = c;
      for (int32_t i = c + 1; i < bs; i++)
        if (fabs(M[i * bs + c]) > fabs(M[piv * bs + c])) piv = i;
      if (!(fabs(M[piv * bs + c]) > 0.0)) {
        rc = -1;
        break;
      }
      for (int32_t j = 0; j < bs && piv != c; j++) {
        double t = M[c * bs + j];
        M[c * bs + j] = M[piv * bs + j];
        M[piv * bs + j] = t;
        t = I[c * bs + j];
        I[c * bs + j] = I[piv * bs + j];
        I[piv * bs + j] = t;
      }
      const double inv = 1.0 / M[c * bs + c];
      for (int32_t j = 0; j < bs; j++) {
        M[c * bs + j] *= inv;
        I[c * bs + j] *= inv;
      }
      for (int32_t i = 0; i < bs; i++) {
        const double f = M[i * bs + c];
        if (i == c || f == 0.0) continue;
        for (int32_t j = 0; j < bs; j++) {
          M[i * bs + j] -= f * M[c * bs + j];
          I[i * bs + j] -= f * I[c * bs + j];
        }
      }
    }
    for (int32_t i = 0; i < bs * bs; i++) minv[b * bs * bs + i] = I[i];
  }
  free(M);
  return rc;
}

/* Preconditioned CG in FP64 (x0 given), M^{-1} = block-Jacobi with blocks of
 * bs rows (bs = 1: Jacobi); stops at ||r|| <= tol ||b||.  Returns the
 * iteration count, or -1 when a diagonal block is singular. */
int32_t orc_pcg(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, const double *b,
                double *x, double tol, int32_t max_iters, int32_t bs) {
  const int64_t nb = ((int64_t)n + bs - 1) / bs;
  double *minv = (double *)malloc(sizeof(double) * nb * bs * bs);
  if (orc_block_jacobi(n, rowPtr, colIdx, val, bs, minv) != 0) {
    free(minv);
    return -1;
  }
  double *r = (double *)calloc((size_t)nb * bs, sizeof(double)), *z = (double *)calloc((size_t)nb * bs, sizeof(double));
  double *p = (double *)malloc(sizeof(double) * n), *q = (double *)malloc(sizeof(double) * n);
  orc_spmv_f64_i32(n, rowPtr, colIdx, val, x, q);
  double bb = 0, rr = 0, rz = 0;
  for (int32_t i = 0; i < n; i++) {
    r[i] = b[i] - q[i];
    bb += b[i] * b[i];
    rr += r[i] * r[i];
  }
#define ORC_APPLY_MINV()                                                   \
  do {                                                                     \
    rz = 0;                                                                \
    for (int64_t blk = 0; blk < nb; blk++)                                 \
      for (int32_t i = 0; i < bs; i++) {                                   \
        double acc = 0;                                                    \
        for (int32_t j = 0; j < bs; j++)                                   \
          acc += minv[blk * bs * bs + i * bs + j] * r[blk * bs + j];       \
        z[blk * bs + i] = acc;                                             \
      }                                                                    \
    for (int32_t i = 0; i < n; i++) rz += r[i] * z[i];                     \
  } while (0)
  ORC_APPLY_MINV();
  for (int32_t i = 0; i < n; i++) p[i] = z[i];
  int32_t it = 0;
  while (it < max_iters && rr > tol * tol * bb) {
    orc_spmv_f64_i32(n, rowPtr, colIdx, val, p, q);
    double pq = 0;
    for (int32_t i = 0; i < n; i++) pq += p[i] * q[i];
    const double a = rz / pq;
    rr = 0;
    for (int32_t i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * q[i];
      rr += r[i] * r[i];
    }
    const double rz_old = rz;
    ORC_APPLY_MINV();
    const double bt = rz / rz_old;
    for (int32_t i = 0; i < n; i++) p[i] = z[i] + bt * p[i];
    it++;
  }
#undef ORC_APPLY_MINV
  free(minv);
  free(r);
  free(z);
  free(p);
  free(q);
  return it;
}

int32_t orc_cg(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, const double *b,
               double *x, double tol, int32_t max_iters) {
  double *r = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
  double *q = (double *)malloc(sizeof(double) * n);
  orc_spmv_f64_i32(n, rowPtr, colIdx, val, x, q);
  double rr = 0, bb = 0;
  for (int32_t i = 0; i < n; i++) {
    r[i] = b[i] - q[i];
    p[i] = r[i];
    rr += r[i] * r[i];
    bb += b[i] * b[i];
  }
  int32_t it = 0;
  while (it < max_iters && rr > tol * tol * bb) {
    orc_spmv_f64_i32(n, rowPtr, colIdx, val, p, q);
    double pq = 0;
    for (int32_t i = 0; i < n; i++) pq += p[i] * q[i];
    const double a = rr / pq;
    double rn = 0;
    for (int32_t i = 0; i < n; i++) {
      x[i] += a * p[i];
      r[i] -= a * q[i];
      rn += r[i] * r[i];
    }
    const double bt = rn / rr;
    for (int32_t i = 0; i < n; i++) p[i] = r[i] + bt * p[i];
    rr = rn;
    it++;
  }
  free(r);
  free(p);
  free(q);
  return it;
}
