// extern "C" wrappers around the reference's own host code, compiled from
// the reference sources (src/ref.cpp, include/dbsr.h, utils/utils.hpp) into
// oracle/_ref/libref_host.so by oracle/Makefile.  TEST INFRASTRUCTURE ONLY:
// it pins the oracle restatement (oracle.c) and generates the golden
// fixtures; the library never loads it.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "matrixFormat.hpp"
#include "ref.h"
#include "dbsr.h"     // csrTodbsr / balanceDbsr / csrTodbsrWithRecorder (non-inline, defined here once)
#include "utils.hpp"  // csrToBcsr<T,Y>

extern "C" {

void ref_spmv_fp64_c(int64_t *rowPtr, int64_t *colIdx, double *val, double *x, double *y, int64_t rows,
                     int64_t cols) {
  double t = 0;
  ref_spmv_fp64(rowPtr, colIdx, val, x, y, rows, cols, t);
}

void ref_spmv_fp32_c(int32_t *rowPtr, int32_t *colIdx, float *val, float *x, float *y, int32_t rows,
                     int32_t cols) {
  ref_spmv_fp32(rowPtr, colIdx, val, x, y, rows, cols);
}

void ref_spmv_fp16_c(int32_t *rowPtr, int32_t *colIdx, float *val, float *x, float *y, int32_t rows,
                     int32_t cols) {
  ref_spmv_fp16(rowPtr, colIdx, val, x, y, rows, cols);
}

struct ref_bcsr_out {
  int32_t rowRegions, colRegions, nonzeroBlocks, blockNum;
  int32_t *rowPtr;   // [rowRegions+1]
  int32_t *colIdx;   // [nonzeroBlocks]
  int32_t *mapping;  // [rowRegions*colRegions]
  double *values;    // [nonzeroBlocks*tm*tk]
};

// csrToBcsr (utils/utils.hpp:10-123); arrays are the reference's own
// allocations, released with ref_free.
void ref_csr2bcsr_c(int32_t rows, int32_t cols, int32_t nnz, int32_t *rowPtr, int32_t *colIdx, double *val,
                    int32_t tm, int32_t tk, ref_bcsr_out *out) {
  CSRFormat<double, int32_t> csr;
  csr.row = rows;
  csr.col = cols;
  csr.nnz = nnz;
  csr.rowPtr = rowPtr;
  csr.colIdx = colIdx;
  csr.values = val;
  BCSRFormat<double, int32_t> b;
  memset(&b, 0, sizeof(b));
  b.TILE_M = tm;
  b.TILE_K = tk;
  b.TILE_N = tk;
  csrToBcsr<double, int32_t>(&csr, &b);
  out->rowRegions = b.rowRegions;
  out->colRegions = b.colRegions;
  out->nonzeroBlocks = b.nonzeroBlocks;
  out->blockNum = b.blockNum;
  out->rowPtr = b.bcsrRowPtr;
  out->colIdx = b.bcsrcolIdx;
  out->mapping = b.relativeBlockIndexMapping;
  out->values = b.values;
}

struct ref_dbsr_out {
  int32_t row, col, nnz, blc_row, blocknnz, warpnum;
  int32_t *blcPtr;       // [blc_row+1]
  int32_t *colIdx;       // [blocknnz]
  double *blcVal;        // [blocknnz]
  uint16_t *blcMap;      // [blocknnz/16]
  int32_t *recorderMap;  // [row] (recorder variant only)
  int32_t *prefix;       // [warpnum+1]
};

static void fill_dbsr(const dbsrMat &d, ref_dbsr_out *out) {
  out->row = d.row;
  out->col = d.col;
  out->nnz = d.nnz;
  out->blc_row = d.blc_row;
  out->blocknnz = d.blocknnz;
  out->warpnum = d.warpnum;
  out->blcPtr = d.blcPtr;
  out->colIdx = d.colIdx;
  out->blcVal = d.blcVal;
  out->blcMap = d.blcMap;
  out->prefix = d.prefix;
}

// csrTodbsrWithRecorder (include/dbsr.h:208-253): stable row sort by length,
// csrTodbsr, balanceDbsr.  balanceDbsr indexes past its warp vector for many
// inputs (its second loop starts from the first loop's leftover fill and
// never reloads it after opening a warp, dbsr.h:139-155); callers only use
// this entry on inputs whose warp walk stays in bounds.
void ref_csr2dbsr_recorder_c(int32_t rows, int32_t cols, int32_t nnz, int32_t *rowPtr, int32_t *colIdx,
                             double *val, ref_dbsr_out *out) {
  CSRFormat<double, int32_t> csr;
  csr.row = rows;
  csr.col = cols;
  csr.nnz = nnz;
  csr.rowPtr = rowPtr;
  csr.colIdx = colIdx;
  csr.values = val;
  dbsrMat d;
  memset(&d, 0, sizeof(d));
  csrTodbsrWithRecorder(&csr, &d);
  fill_dbsr(d, out);
  out->recorderMap = d.recorderMap;
}

// csrRecorderSelf (include/dbsr.h:170-206): rows stably sorted by length.
void ref_recorder_self_c(int32_t rows, int32_t cols, int32_t nnz, int32_t *rowPtr, int32_t *colIdx, double *val,
                         int32_t **outRowPtr, int32_t **outColIdx, double **outVal) {
  CSRFormat<double, int32_t> csr, re;
  csr.row = rows;
  csr.col = cols;
  csr.nnz = nnz;
  csr.rowPtr = rowPtr;
  csr.colIdx = colIdx;
  csr.values = val;
  csrRecorderSelf(&csr, &re);
  *outRowPtr = re.rowPtr;
  *outColIdx = re.colIdx;
  *outVal = re.values;
}

// csrTodbsr alone (include/dbsr.h:10-92).
void ref_csr2dbsr_c(int32_t rows, int32_t cols, int32_t nnz, int32_t *rowPtr, int32_t *colIdx, double *val,
                    ref_dbsr_out *out) {
  CSRFormat<double, int32_t> csr;
  csr.row = rows;
  csr.col = cols;
  csr.nnz = nnz;
  csr.rowPtr = rowPtr;
  csr.colIdx = colIdx;
  csr.values = val;
  dbsrMat d;
  memset(&d, 0, sizeof(d));
  csrTodbsr(&csr, &d);
  fill_dbsr(d, out);
  out->recorderMap = nullptr;
  out->prefix = nullptr;
  out->warpnum = 0;
}

// balanceDbsr alone (include/dbsr.h:94-168) on a block-row pointer; see the
// bounds note above.
void ref_balance_dbsr_c(int32_t row, int32_t col, int32_t nnz, int32_t blc_row, int32_t *blcPtr,
                        int32_t *warpnum, int32_t **prefix) {
  dbsrMat d;
  memset(&d, 0, sizeof(d));
  d.row = row;
  d.col = col;
  d.nnz = nnz;
  d.blc_row = blc_row;
  d.blcPtr = blcPtr;
  balanceDbsr(&d);
  *warpnum = d.warpnum;
  *prefix = d.prefix;
}

void ref_free(void *p) { free(p); }

}  // extern "C"
