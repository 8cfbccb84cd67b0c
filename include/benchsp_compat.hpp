/*
 * benchsp_compat.hpp — the reference's C++ operator surface (jiajun-c/benchsp
 * include/csrspmv.h, spmv.h, amgT.h, bcsr.h, dasp.h, smat.h, cusp.h) with the
 * same names, signatures and C++ linkage, implemented in
 * libbspmv_compat.so on top of the C ABI of libbspmv (bsp.h).  A program
 * written against the reference's headers links unchanged against
 * libbspmv_compat.so + libbspmv.so.
 *
 * Semantics kept from the reference: host pointers in and out; the call
 * uploads, runs `repeat` timed launches (each followed by a device
 * synchronize, timed on the host clock like the reference's std::chrono
 * loops) and downloads the result; avg_time is microseconds per launch
 * (the reference truncates it to whole microseconds; here it is fractional);
 * spmv_all returns Y in order_rid order and fills order_rid; the DBSR calls
 * return y in the DBSR's (recorder) row order.
 *
 * Deliberate differences, where the reference's result is not A*x:
 *  - y is overwritten with A*x.  The reference's AmgT, DBSR and CSR-balance
 *    kernels add into y with atomics across all warm-up and timed launches
 *    (src/amgT.cu, src/csrspmv.cu:59-102); bsp_compat_set_accumulate(1)
 *    gives y_out = y_in + A*x instead (added once).
 *  - The DBSR kernels compute A*x; the reference multiplies by a B fragment
 *    of ones and so returns row sums (src/amgT.cu:356, :425).
 *  - MySpmvWithPrefp64 stores y in double (the reference rounds it to float,
 *    src/spmv.cu:395).
 *  - smatSpmmfp16 writes C = A * ones(col x n) (FP32 accumulation) into
 *    outvalues, row-major row x n; the reference never writes outvalues.
 *  - cusparse_spmv reads the int64 column array as int64 (the reference
 *    passes it to cuSPARSE as 32-bit indices, src/cusparse.cu:69);
 *    cusparse_spmv_fp16 passes FP32 alpha/beta for its FP32 compute type.
 *  - MySpmvWithPre, declared but never defined by the reference, is an FP32
 *    SpMV.
 * Errors print bsp_last_error() to stderr; int functions return 1 (the
 * reference exits the process through its CHECK macro).
 */
#ifndef BENCHSP_COMPAT_HPP
#define BENCHSP_COMPAT_HPP

#include <cuda_fp16.h>
#include <stdint.h>

/* Layout of the reference's dbsrMat (include/matrixFormat.hpp:86-106):
 * host arrays as built by its csrTodbsr / csrTodbsrWithRecorder. */
class dbsrMat {
 public:
  int row;
  int col;
  int nnz;
  int blc_row;
  int blc_col;
  int blc_num;
  double stand;
  double avg_nnz;
  int32_t *blcPtr;
  int32_t *colIdx;
  double *blcVal;
  unsigned short *blcMap;
  int32_t blocknnz;
  int32_t warpnum;
  int32_t *rowPtrbyWarp;
  int32_t *rowIdxbyWarp;
  int32_t *recorderMap;
  int32_t *prefix;
};

/* include/csrspmv.h:2-3 (src/csrspmv.cu:104, :136) */
int spmv_fp64_warpper(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz, double *values,
                      double *x, double *outvalues, int repeat, double &avg_time);
int spmv_fp64_balance_warpper(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz,
                              double *values, double *x, double *outvalues, int repeat, double &avg_time);

/* include/spmv.h:1-3 (src/spmv.cu:197, :323) */
void MySpmvWithPre(int *rowPtr, int *colIdx, int rows, int cols, int nnz, float *values, float *x,
                   float *outvalues);
void MySpmvWithPrefp16(int32_t *rowPtr, int32_t *colIdx, int32_t rows, int32_t cols, int32_t nnz, float *values,
                       float *x, float *outvalues);
void MySpmvWithPrefp64(int64_t *rowPtr, int64_t *colIdx, int64_t rows, int64_t cols, int64_t nnz, double *values,
                       double *x, double *outvalues);

/* include/amgT.h:3-6 (src/amgT.cu:1355, :1280, :1202) */
int amgT_spmv_fp64(int32_t *hA_csrOffsets, int32_t *hA_columns, double *hA_values, double *hX, double *hY,
                   int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz, int repeat, double &avg_time);
int amgT_spmv_fp64_dbsr(dbsrMat *dbsr, double *hX, double *hY, int32_t warmup, int32_t repeat, double &avg_time);
int amgT_spmv_fp64_dbsr_balance(dbsrMat *dbsr, double *hX, double *hY, int32_t warmup, int32_t repeat,
                                double &avg_time);

/* include/bcsr.h:3 (src/bcsr.cu:224): 3x3 tiles, as the reference uses */
void bcsr_spmv_fp64(int64_t *hA_csrOffsets, int64_t *hA_columns, double *hA_values32, double *hX32,
                    double *hY32, int64_t A_num_rows, int64_t A_num_cols, int64_t A_nnz, int repeat);

/* include/dasp.h:1-2 (src/dasp.cu:814); filename and NUM are unused, as in
 * the reference */
void spmv_all(char *filename, double *csrValA, int *csrRowPtrA, int *csrColIdxA, double *X_val, double *Y_val,
              int *order_rid, int rowA, int colA, int nnzA, int NUM, double threshold, int block_longest,
              double &avg_time);

/* include/smat.h:1 (src/smat.cu:103) */
void smatSpmmfp16(int *rowPtr, int *colIdx, int row, int col, int n, int nnz, float *values, float *outvalues);

/* include/cusp.h:3-6 (src/cusparse.cu:35, :104, :200, and the FP16
 * wrapper): cuSPARSE, for comparison only */
int cusparse_spmv(int *A_csrOffsets, int64_t *A_columns, float *A_values, float *x, float *y, int64_t row,
                  int64_t col, int64_t nnz);
int cusparse_spmv_fp64(int64_t *hA_csrOffsets, int64_t *hA_columns, double *hA_values, double *hX, double *hY,
                       int64_t A_num_rows, int64_t A_num_cols, int64_t A_nnz, int repeat, double &avg_time);
int cusparse_spmv_fp16(int *hA_csrOffsets, int32_t *hA_columns, half *hA_values, half *hX, half *hY,
                       int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz);
void cusparse_spmv_fp16_warpper(int *hA_csrOffsets, int32_t *hA_columns, float *hA_values32, float *hX32,
                                float *hY32, int32_t A_num_rows, int32_t A_num_cols, int32_t A_nnz);

/* Compat switches (no reference counterpart). */
extern "C" void bsp_compat_set_accumulate(int on); /* y_out = y_in + A*x */
extern "C" int bsp_compat_get_accumulate(void);

#endif /* BENCHSP_COMPAT_HPP */
