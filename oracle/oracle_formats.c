/*
 * oracle_formats.c — CPU restatement of the reference's format converters
 * (BCSR, DBSR, block statistics).  TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include <math.h>
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

/* ---- DASP packing (src/dasp.cu:827-1482) ------------------------------- */

static int32_t *i32z(int64_t n) { return (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t)); }
static double *f64z(int64_t n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* Stable sort of row ids by length, descending (radix_sort with the
 * descending count_sort, dasp.cu:214-246, :282-289). */
static void sort_desc_stable(int32_t *len, int32_t *rid, int32_t n) {
  int32_t mx = 0;
  for (int32_t i = 0; i < n; i++)
    if (len[i] > mx) mx = len[i];
  int32_t *cnt = i32z((int64_t)mx + 2);
  int32_t *l2 = i32z(n), *r2 = i32z(n);
  for (int32_t i = 0; i < n; i++) cnt[mx - len[i]]++;
  int32_t acc = 0;
  for (int32_t k = 0; k <= mx; k++) {
    const int32_t c = cnt[k];
    cnt[k] = acc;
    acc += c;
  }
  for (int32_t i = 0; i < n; i++) {
    const int32_t p = cnt[mx - len[i]]++;
    l2[p] = len[i];
    r2[p] = rid[i];
  }
  memcpy(len, l2, sizeof(int32_t) * (size_t)n);
  memcpy(rid, r2, sizeof(int32_t) * (size_t)n);
  free(cnt);
  free(l2);
  free(r2);
}

void orc_dasp_pack(int32_t rows, const int32_t *rp, const int32_t *ci, const double *va, double threshold,
                   int32_t block_longest, orc_dasp *o) {
  memset(o, 0, sizeof(*o));
  int32_t n1 = 0, n2 = 0, n3 = 0, n4 = 0, nl = 0, nb = 0, nz = 0;
  for (int32_t i = 0; i < rows; i++) {  /* dasp.cu:827-859 */
    const int32_t len = rp[i + 1] - rp[i];
    if (len == 1) n1++;
    else if (len == 3) n3++;
    else if (len == 2) n2++;
    else if (len == 0) nz++;
    else if (len == 4) n4++;
    else if (len >= block_longest) nl++;
    else nb++;
  }
  int32_t *r1 = i32z(n1), *r2 = i32z(n2), *r3 = i32z(n3), *r4 = i32z(n4), *rl = i32z(nl), *rz = i32z(nz);
  int32_t *rb = i32z(nb), *lb = i32z((int64_t)nb + 1), *ll = i32z((int64_t)nl + 1);
  int32_t k1 = 0, k2 = 0, k3 = 0, k4 = 0, kl = 0, kb = 0, kz = 0;
  for (int32_t i = 0; i < rows; i++) {  /* dasp.cu:876-918 */
    const int32_t len = rp[i + 1] - rp[i];
    if (len == 1) r1[k1++] = i;
    else if (len == 3) r3[k3++] = i;
    else if (len == 2) r2[k2++] = i;
    else if (len == 0) rz[kz++] = i;
    else if (len == 4) r4[k4++] = i;
    else if (len >= block_longest) { ll[kl] = len; rl[kl++] = i; }
    else { lb[kb] = len; rb[kb++] = i; }
  }
  int32_t c13 = n1 < n3 ? n1 : n3;  /* dasp.cu:922-933 */
  if (c13 / 8 >= 16) c13 = 8 * (c13 / 8);
  else c13 = 0;
  const int32_t s1 = n1 - c13, s3 = n3 - c13, s34 = s3 + n4;
  const int32_t sb13 = (c13 + 7) / 8, sb22 = ((n2 + 1) / 2 + 7) / 8, sb34 = (s34 + 7) / 8;
  const int32_t tb13 = (sb13 + 7) / 8, tb22 = (sb22 + 7) / 8, tb34 = (sb34 + 15) / 16;
  const int32_t f13 = tb13 * 8 * 32, f34 = tb34 * 16 * 32, f22 = tb22 * 8 * 32;
  const int32_t fs = s1 + f13 + f34 + f22;
  o->row_long = nl; o->row_block = nb; o->row_zero = nz; o->short_row_1 = s1; o->short_row_2 = n2;
  o->short_row_3 = s3; o->short_row_4 = n4; o->common_13 = c13; o->short_row_34 = s34;
  o->fill0_nnz_short13 = f13; o->fill0_nnz_short34 = f34; o->fill0_nnz_short = fs;
  o->short_val = f64z(fs);
  o->short_cid = i32z(fs);
  for (int32_t i = 0; i < s1; i++) {  /* dasp.cu:961-966 */
    o->short_val[i] = va[rp[r1[i]]];
    o->short_cid[i] = ci[rp[r1[i]]];
  }
  for (int32_t i = 0; i < sb13; i++)  /* dasp.cu:968-988 */
    for (int32_t j = 0; j < 8 && i * 8 + j < c13; j++) {
      const int64_t b = s1 + (int64_t)i * 32 + j * 4;
      const int32_t a = rp[r1[s1 + i * 8 + j]], c = rp[r3[i * 8 + j]];
      o->short_val[b] = va[a];
      o->short_cid[b] = ci[a];
      for (int t = 0; t < 3; t++) {
        o->short_val[b + 1 + t] = va[c + t];
        o->short_cid[b + 1 + t] = ci[c + t];
      }
    }
  for (int32_t i = 0; i < s3; i++) {  /* dasp.cu:990-1005 */
    const int64_t b = s1 + f13 + (int64_t)i * 4;
    const int32_t c = rp[r3[c13 + i]];
    for (int t = 0; t < 3; t++) {
      o->short_val[b + t] = va[c + t];
      o->short_cid[b + t] = ci[c + t];
    }
  }
  for (int32_t i = 0; i < n4; i++) {  /* dasp.cu:1007-1021 */
    const int64_t b = s1 + f13 + ((int64_t)s3 + i) * 4;
    const int32_t c = rp[r4[i]];
    for (int t = 0; t < 4; t++) {
      o->short_val[b + t] = va[c + t];
      o->short_cid[b + t] = ci[c + t];
    }
  }
  for (int32_t i = 0; i < sb22; i++)  /* dasp.cu:1023-1038 */
    for (int32_t j = 0; j < 16 && i * 16 + j < n2; j++) {
      const int64_t b = s1 + f13 + f34 + (int64_t)i * 32 + (j % 8) * 4 + (j / 8) * 2;
      const int32_t c = rp[r2[i * 16 + j]];
      o->short_val[b] = va[c];
      o->short_val[b + 1] = va[c + 1];
      o->short_cid[b] = ci[c];
      o->short_cid[b + 1] = ci[c + 1];
    }
  sort_desc_stable(lb, rb, nb);  /* dasp.cu:1244 */
  /* long rows (dasp.cu:1326-1369) */
  o->long_ptr_warp = i32z((int64_t)nl + 1);
  for (int32_t i = 0; i < nl; i++) o->long_ptr_warp[i + 1] = o->long_ptr_warp[i] + (ll[i] + 63) / 64;
  const int32_t lw = o->long_ptr_warp[nl];
  const int32_t bnl = (lw + 3) / 4;
  o->fill0_nnz_long = bnl * 4 * 64;
  o->long_val = f64z(o->fill0_nnz_long);
  o->long_cid = i32z(o->fill0_nnz_long);
  for (int32_t i = 0; i < nl; i++)
    for (int32_t j = 0; j < ll[i]; j++) {
      o->long_val[(int64_t)o->long_ptr_warp[i] * 64 + j] = va[rp[rl[i]] + j];
      o->long_cid[(int64_t)o->long_ptr_warp[i] * 64 + j] = ci[rp[rl[i]] + j];
    }
  /* row-block part (dasp.cu:1374-1482), rowloop = 1 */
  int32_t blocknum = (nb + 7) / 8;
  blocknum = ((blocknum + 3) / 4) * 4;
  o->blocknum = blocknum;
  o->block_ptr = i32z((int64_t)blocknum + 1);
  o->irreg_rpt = i32z((int64_t)nb + 1);
  for (int32_t i = 0; i < blocknum; i++) {
    const int32_t rs = i * 8, re = (i + 1) * 8 >= nb ? nb : (i + 1) * 8;
    for (int32_t k = 1;; k++) {
      int32_t block_nnz = 0;
      for (int32_t r = rs; r < re; r++) {
        if (lb[r] / 4 >= k) block_nnz += 4;
        else if (lb[r] / 4 == k - 1) block_nnz += lb[r] % 4;
      }
      if (block_nnz >= threshold * 4 * 8) {
        o->block_ptr[i] += 32;
      } else {
        for (int32_t r = rs; r < re; r++) o->irreg_rpt[r] = lb[r] - (k - 1) * 4 > 0 ? lb[r] - (k - 1) * 4 : 0;
        break;
      }
    }
  }
  for (int32_t i = 0, acc = 0; i <= blocknum; i++) {
    const int32_t c = o->block_ptr[i];
    o->block_ptr[i] = acc;
    acc += c;
  }
  for (int32_t i = 0, acc = 0; i <= nb; i++) {
    const int32_t c = o->irreg_rpt[i];
    o->irreg_rpt[i] = acc;
    acc += c;
  }
  o->fill0_nnz_reg = o->block_ptr[blocknum];
  o->nnz_irreg = o->irreg_rpt[nb];
  o->irreg_val = f64z(o->nnz_irreg);
  o->irreg_cid = i32z(o->nnz_irreg);
  for (int32_t i = 0; i < nb; i++) {
    const int32_t off = o->irreg_rpt[i], n = o->irreg_rpt[i + 1] - off, end = rp[rb[i] + 1];
    for (int32_t j = 0; j < n; j++) {
      o->irreg_val[off + j] = va[end - n + j];
      o->irreg_cid[off + j] = ci[end - n + j];
    }
  }
  o->reg_val = f64z(o->fill0_nnz_reg);
  o->reg_cid = i32z(o->fill0_nnz_reg);
  for (int32_t b = 0; b < blocknum; b++) {
    const int32_t blocklen = (o->block_ptr[b + 1] - o->block_ptr[b]) / 8;
    for (int32_t r = 0; r < 8; r++) {
      const int32_t row = b * 8 + r;
      for (int32_t i = 0; i < blocklen; i++) {
        /* pre-layout index r*blocklen+i re-laid to tile-major (:1477-1482) */
        const int64_t dst = o->block_ptr[b] + (i / 4) * 32 + r * 4 + i % 4;
        if (row < nb && i < lb[row]) {
          o->reg_val[dst] = va[rp[rb[row]] + i];
          o->reg_cid[dst] = ci[rp[rb[row]] + i];
        }
      }
    }
  }
  /* order_rid (dasp.cu:1289-1306) */
  o->order_rid = i32z(rows);
  int64_t p = 0;
  for (int32_t i = 0; i < nl; i++) o->order_rid[p++] = rl[i];
  for (int32_t i = 0; i < nb; i++) o->order_rid[p++] = rb[i];
  for (int32_t i = 0; i < s1; i++) o->order_rid[p++] = r1[i];
  for (int32_t i = 0; i < sb13; i++) {
    for (int32_t j = 0; j < 8; j++) o->order_rid[p + j] = r1[s1 + i * 8 + j];
    for (int32_t j = 0; j < 8; j++) o->order_rid[p + 8 + j] = r3[i * 8 + j];
    p += 16;
  }
  for (int32_t i = 0; i < s3; i++) o->order_rid[p++] = r3[c13 + i];
  for (int32_t i = 0; i < n4; i++) o->order_rid[p++] = r4[i];
  for (int32_t i = 0; i < n2; i++) o->order_rid[p++] = r2[i];
  for (int32_t i = 0; i < nz; i++) o->order_rid[p++] = rz[i];
  /* the kernel's block ranges (dasp.cu:1513-1539) */
  o->offset_reg = bnl;
  o->offset_short1 = bnl + blocknum / 4;
  o->offset_short13 = o->offset_short1 + (s1 + 127) / 128;
  o->offset_short34 = o->offset_short13 + tb13;
  o->offset_short22 = o->offset_short34 + tb34;
  o->block_num_all = o->offset_short22 + tb22;
  free(r1); free(r2); free(r3); free(r4); free(rl); free(rz); free(rb); free(lb); free(ll);
}

void orc_dasp_free(orc_dasp *o) {
  free(o->short_val); free(o->short_cid); free(o->long_val); free(o->long_cid); free(o->long_ptr_warp);
  free(o->reg_val); free(o->reg_cid); free(o->block_ptr); free(o->irreg_val); free(o->irreg_cid);
  free(o->irreg_rpt); free(o->order_rid);
  memset(o, 0, sizeof(*o));
}

/* ---- Block statistics (bench/blockinfo.cpp:96-119) --------------------- */

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

static int64_t distinct_u32(uint32_t *k, int64_t n) {
  qsort(k, (size_t)n, sizeof(uint32_t), cmp_u32);
  int64_t c = 0;
  for (int64_t i = 0; i < n; i++) c += (i == 0 || k[i] != k[i - 1]);
  return c;
}

void orc_blockinfo(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, int64_t *blocks,
                   int64_t *blocks_recorder) {
  /* keys row/4*1000005 + col/4 and row/4*1000005 + z/4 in wrapping 32-bit
   * arithmetic, as the reference's int expressions evaluate */
  const int64_t nnz = rowPtr[rows];
  uint32_t *kp = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nnz > 0 ? nnz : 1));
  uint32_t *kr = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nnz > 0 ? nnz : 1));
  for (int32_t r = 0; r < rows; r++)
    for (int32_t j = rowPtr[r]; j < rowPtr[r + 1]; j++) {
      const uint32_t base = (uint32_t)(r / 4) * 1000005u;
      kp[j] = base + (uint32_t)(colIdx[j] / 4);
      kr[j] = base + (uint32_t)((j - rowPtr[r]) / 4);
    }
  *blocks = distinct_u32(kp, nnz);
  *blocks_recorder = distinct_u32(kr, nnz);
  free(kp);
  free(kr);
}

/* ------------------------------------------------------------------------
 * Per-block power-of-two-scaled FP16/BF16 BSR (the format of the library's
 * bsp_bsr_scaled; the reference has no scaled storage, its BSR values are
 * FP64 only, src/amgT.cu:210-274).  Per block: m = max |a|, E = floor(log2 m)
 * from the exponent bits, e = E - 14 (FP16: the largest magnitude lands in
 * [2^14, 2^15)) or E (BF16: [1, 2)), clamped to [-126, 127], e = 0 for an
 * all-zero block; q = round-to-nearest-even((float)(a * 2^-e)).  Values are
 * stored in 4x4 tiles (row-major inside a tile; an 8x8 block's tiles in the
 * order (0,0), (0,1), (1,0), (1,1)); key = block column | (e + 128) << 24.
 * Returns 1 when a value is not finite or rounds to inf, else 0. */
int32_t orc_bsr_scale(int64_t nb, int32_t bs, int32_t dtype, const int32_t *blcIdx, const double *blcVal,
                      uint32_t *key, uint16_t *val) {
  int32_t bad = 0;
  const int bb = bs * bs, ts = bs / 4;
  for (int64_t k = 0; k < nb; k++) {
    const double *v = blcVal + k * bb;
    double m = 0;
    for (int i = 0; i < bb; i++) {
      const double a = fabs(v[i]);
      if (!(a <= 1.7976931348623157e308)) bad = 1;
      if (a > m) m = a;
    }
    int e = 0;
    if (m > 0) {
      uint64_t bits;
      memcpy(&bits, &m, 8);
      const int E = (int)((bits >> 52) & 0x7ff) - 1023;
      e = dtype == 2 ? E - 14 : E; /* 2 = FP16, 3 = BF16 */
      if (e < -126) e = -126;
      if (e > 127) e = 127;
    }
    const double down = ldexp(1.0, -e);
    for (int r = 0; r < bs; r++)
      for (int c = 0; c < bs; c++) {
        const float f = (float)(v[r * bs + c] * down);
        uint16_t q;
        if (dtype == 2) {
          q = orc_f32_to_f16(f);
          if ((q & 0x7c00u) == 0x7c00u) bad = 1;
        } else {
          q = orc_f32_to_bf16(f);
          if ((q & 0x7f80u) == 0x7f80u) bad = 1;
        }
        const int t = (r / 4) * ts + c / 4;
        val[k * bb + t * 16 + (r % 4) * 4 + c % 4] = q;
      }
    key[k] = (uint32_t)blcIdx[k] | ((uint32_t)(e + 128) << 24);
  }
  return bad;
}

/* The scaled blocks back to FP64 in row-major block order (exact: q times a
 * power of two). */
void orc_bsr_unscale(int64_t nb, int32_t bs, int32_t dtype, const uint32_t *key, const uint16_t *val, double *out) {
  const int bb = bs * bs, ts = bs / 4;
  for (int64_t k = 0; k < nb; k++) {
    const int e = (int)(key[k] >> 24) - 128;
    for (int r = 0; r < bs; r++)
      for (int c = 0; c < bs; c++) {
        const uint16_t q = val[k * bb + ((r / 4) * ts + c / 4) * 16 + (r % 4) * 4 + c % 4];
        const double f = dtype == 2 ? (double)orc_f16_to_f32(q) : (double)orc_bf16_to_f32(q);
        out[k * bb + r * bs + c] = ldexp(f, e);
      }
  }
}
