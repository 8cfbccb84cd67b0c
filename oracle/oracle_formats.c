/*
 * oracle_formats.c — CPU restatement of the reference's format converters
 * (BCSR, DBSR, block statistics).  TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- DBSR (include/dbsr.h) -------------------------------------------- */

typedef struct {
  int32_t len, row;
} len_row;

static int cmp_len_row(const void *a, const void *b) {
  const len_row *x = (const len_row *)a, *y = (const len_row *)b;
  if (x->len != y->len) return (x->len > y->len) - (x->len < y->len);
  return (x->row > y->row) - (x->row < y->row);
}

void orc_recorder(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t *order,
                  int32_t *newPtr, int32_t *newCol, double *newVal) {
  /* csrRecorderSelf / csrTodbsrWithRecorder (dbsr.h:170-206, :208-233):
   * std::sort of (len, row) pairs, then rows gathered in that order */
  len_row *lr = (len_row *)malloc(sizeof(len_row) * (rows > 0 ? rows : 1));
  for (int32_t i = 0; i < rows; i++) {
    lr[i].len = rowPtr[i + 1] - rowPtr[i];
    lr[i].row = i;
  }
  qsort(lr, (size_t)rows, sizeof(len_row), cmp_len_row);
  newPtr[0] = 0;
  for (int32_t k = 0; k < rows; k++) {
    order[k] = lr[k].row;
    newPtr[k + 1] = newPtr[k] + lr[k].len;
    const int32_t s = rowPtr[lr[k].row];
    for (int32_t j = 0; j < lr[k].len; j++) {
      newCol[newPtr[k] + j] = colIdx[s + j];
      newVal[newPtr[k] + j] = val[s + j];
    }
  }
  free(lr);
}

int32_t orc_dbsr_blocks(int32_t rows, const int32_t *rowPtr, int32_t *blcPtr) {
  /* csrTodbsr, block pointer (dbsr.h:18-26) */
  const int32_t brow = (rows + 3) / 4;
  if (blcPtr) memset(blcPtr, 0, sizeof(int32_t) * (brow + 1));
  int32_t total = 0;
  for (int32_t b = 0; b < brow; b++) {
    int32_t m = 0;
    for (int32_t i = 4 * b; i < 4 * b + 4 && i < rows; i++) {
      const int32_t c = (rowPtr[i + 1] - rowPtr[i] + 3) / 4;
      if (c > m) m = c;
    }
    if (blcPtr) blcPtr[b] = total;
    total += m;
  }
  if (blcPtr) blcPtr[brow] = total;
  return total;
}

void orc_dbsr_fill(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                   const int32_t *blcPtr, int32_t *outCol, double *outVal, uint16_t *map) {
  /* csrTodbsr, scatter (dbsr.h:65-79); caller zero-fills the outputs */
  for (int32_t i = 0; i < rows; i++) {
    int32_t z = 0;
    for (int32_t j = rowPtr[i]; j < rowPtr[i + 1]; j++, z++) {
      const int64_t blk = blcPtr[i / 4] + z / 4;
      const int pos = (i % 4) * 4 + z % 4;
      outVal[blk * 16 + pos] = val[j];
      outCol[blk * 16 + pos] = colIdx[j];
      map[blk] |= (uint16_t)(1u << pos);
    }
  }
}

int32_t orc_dbsr_balance(int32_t brow, const int32_t *blcPtr, int32_t *prefix, int32_t cap_prefix,
                         int32_t *overflow) {
  /* balanceDbsr (dbsr.h:94-168), both walks as written; the second starts
   * from the first one's leftover fill.  Returns the number of warps (the
   * first walk's count, grown when the second walk runs past it). */
  const int32_t CAP = 64;
  int32_t now = 0, warpcount = 0;
  for (int32_t i = 0; i < brow; i++) {
    const int32_t len = blcPtr[i + 1] - blcPtr[i];
    if (now + len <= CAP) {
      now += len;
    } else {
      if (now != 0) {
        warpcount++;
        now = 0;
      }
      if (len <= CAP)
        now = len;
      else
        warpcount += (len + CAP - 1) / CAP;
    }
  }
  if (now) warpcount++;
  int32_t cap = brow + blcPtr[brow] / CAP + 2;
  int32_t *counts = (int32_t *)calloc((size_t)cap + 1, sizeof(int32_t));
  int32_t now_warp = 0, last = -1;
  for (int32_t i = 0; i < brow; i++) {
    const int32_t len = blcPtr[i + 1] - blcPtr[i];
    if (now + len <= CAP) {
      counts[now_warp]++;
      if (now_warp > last) last = now_warp;
      now += len;
    } else {
      if (now != 0) now = 0;
      if (len <= CAP) {
        now_warp++;
        counts[now_warp]++;
        if (now_warp > last) last = now_warp;
      } else {
        for (int32_t j = 1; j <= (len + CAP - 1) / CAP; j++) {
          now_warp++;
          counts[now_warp]++;
          if (now_warp > last) last = now_warp;
        }
      }
    }
  }
  const int32_t of = last >= warpcount;
  const int32_t warpnum = of ? last + 1 : warpcount;
  if (overflow) *overflow = of;
  if (prefix) {
    prefix[0] = 0;
    for (int32_t w = 0; w < warpnum && w < cap_prefix; w++) prefix[w + 1] = prefix[w] + counts[w];
  }
  free(counts);
  return warpnum;
}

/* ---- BCSR (utils/utils.hpp:10-123) ------------------------------------ */

int64_t orc_csr2bcsr(int32_t rows, int32_t cols, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                     int32_t tm, int32_t tk, int32_t *bRowPtr, int32_t *bColIdx, double *bVal, int32_t *mapping) {
  /* Dense block-occupancy table over rowRegions x colRegions, blocks
   * numbered row-major (relativeBlockIndexMapping), values row-major
   * tm x tk.  Pass 1 (bRowPtr NULL) returns nonzeroBlocks. */
  const int64_t nr = (rows + tm - 1) / tm, nc = (cols + tk - 1) / tk;
  int32_t *info = (int32_t *)calloc((size_t)(nr * nc > 0 ? nr * nc : 1), sizeof(int32_t));
  int64_t nb = 0;
  for (int32_t r = 0; r < rows; r++)
    for (int32_t j = rowPtr[r]; j < rowPtr[r + 1]; j++) {
      const int64_t b = (int64_t)(r / tm) * nc + colIdx[j] / tk;
      if (!info[b]) {
        info[b] = 1;
        nb++;
      }
    }
  if (bRowPtr) {
    int64_t rel = 0;
    for (int64_t b = 0; b < nr * nc; b++) {
      const int32_t m = info[b] ? (int32_t)rel++ : -1;
      if (mapping) mapping[b] = m;
      info[b] = m;
    }
    int64_t k = 0;
    for (int64_t br = 0; br < nr; br++) {
      bRowPtr[br] = (int32_t)k;
      for (int64_t bc = 0; bc < nc; bc++)
        if (info[br * nc + bc] >= 0) bColIdx[k++] = (int32_t)bc;
    }
    bRowPtr[nr] = (int32_t)k;
    memset(bVal, 0, sizeof(double) * (size_t)(nb * tm * tk));
    for (int32_t r = 0; r < rows; r++)
      for (int32_t j = rowPtr[r]; j < rowPtr[r + 1]; j++) {
        const int64_t b = info[(int64_t)(r / tm) * nc + colIdx[j] / tk];
        bVal[b * tm * tk + (r % tm) * tk + colIdx[j] % tk] = val[j];
      }
  }
  free(info);
  return nb;
}
