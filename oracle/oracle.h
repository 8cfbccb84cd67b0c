/*
 * oracle.h — CPU restatement of the reference's (jiajun-c/benchsp) hot-path
 * algorithms.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
 * and the CPU-baseline leg of bench.py use it as the checker.  The library
 * (benchsp_b200, libbspmv.so) never links, loads or calls anything here.
 *
 * Each function cites the reference file:line it restates.  Parity pins:
 * the restatement is checked against the reference's own code compiled
 * from its sources into oracle/_ref (ref.cpp, include/dbsr.h,
 * utils/utils.hpp through g++; src/dasp.cu's packing through a CPU stub
 * of the CUDA runtime) on the committed golden fixtures.
 */
#ifndef BSP_ORACLE_H
#define BSP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y_i = sum_j A_ij x_j, left to right, separately rounded mul and add
 * (src/ref.cpp:26-37). */
void orc_spmv_f64(int64_t rows, const int64_t *rowPtr, const int64_t *colIdx, const double *val,
                  const double *x, double *y);
/* Same on int32 CSR. */
void orc_spmv_f64_i32(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                      const double *x, double *y);
/* FP32 sum (src/ref.cpp:14-24). */
void orc_spmv_f32(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const float *val,
                  const float *x, float *y);
/* FP16 variant (src/ref.cpp:3-13): val/x given as IEEE half bit patterns,
 * float sum of products, result rounded to half (bits returned). */
void orc_spmv_f16(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const uint16_t *val,
                  const uint16_t *x, uint16_t *y);
uint16_t orc_f32_to_f16(float f);  /* round to nearest even */
float orc_f16_to_f32(uint16_t h);
uint16_t orc_f32_to_bf16(float f); /* round to nearest even */
float orc_bf16_to_f32(uint16_t h);

/* |sum_j |A_ij x_j|| per row, the scale of the rounding-error bound used by
 * the parity tests. */
void orc_spmm_f64(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t N,
                  const double *B, double *Cout, double *absC);
void orc_abs_rowsum(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                    const double *x, double *out);

/* FP64 CG with orc_spmv_f64_i32 (the CPU oracle of the GPU solves).  x holds
 * the initial guess on entry and the solution on exit; returns iterations. */
int32_t orc_block_jacobi(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t bs,
                         double *minv);
int32_t orc_pcg(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, const double *b,
                double *x, double tol, int32_t max_iters, int32_t bs);
int32_t orc_cg(int32_t n, const int32_t *rowPtr, const int32_t *colIdx, const double *val, const double *b,
               double *x, double tol, int32_t max_iters);

/* AmgT CSR -> BSR (CSR2BSR_GPU, src/amgT.cu:1114-1172): block columns
 * ascending inside a block-row (rank by counting smaller keys, :823-835),
 * row-major bs x bs values (:840-847), bitmap bit r*bs+c (:776,:836).
 * Pass 1 (arrays NULL) returns blc_num; pass 2 fills caller arrays:
 * blcPtr[blc_row+1], blcIdx[blc_num], blcVal[blc_num*bs*bs], blcMap[blc_num]
 * (uint64 per block, low bs*bs bits). */
int64_t orc_csr2bsr(int32_t rows, int32_t cols, const int32_t *rowPtr, const int32_t *colIdx,
                    const double *val, int32_t bs, int32_t *blcPtr, int32_t *blcIdx, double *blcVal,
                    uint64_t *blcMap);
/* Balanced chunks (get_rowPtrbyWarp / get_rowIdxbyWarp + exclusive scan,
 * src/amgT.cu:523-545, :1174-1200): rowPtrbyWarp[blc_row+1] = exclusive
 * scan of ceil(len/64); rowIdxbyWarp (may be NULL) gets warpnum entries.
 * Returns warpnum. */
int32_t orc_bsr_chunks(int32_t blc_row, const int32_t *blcPtr, int32_t *rowPtrbyWarp, int32_t *rowIdxbyWarp);
/* sqrtf(sum (len - avg)^2 / blc_row) (getStand, src/amgT.cu:546-575, :1146-1155). */
double orc_bsr_stand(int32_t blc_row, const int32_t *blcPtr);

/* DBSR (include/dbsr.h).  orc_recorder: rows stably sorted ascending by
 * length (csrRecorderSelf, :170-206), order[new] = old.  orc_dbsr_blocks:
 * block pointer of csrTodbsr (:18-26), returns the block count.
 * orc_dbsr_fill: its scatter (:65-79) into zero-filled arrays.
 * orc_dbsr_balance: balanceDbsr's two walks (:94-168), prefix[warps+1]. */
void orc_recorder(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val, int32_t *order,
                  int32_t *newPtr, int32_t *newCol, double *newVal);
int32_t orc_dbsr_blocks(int32_t rows, const int32_t *rowPtr, int32_t *blcPtr);
void orc_dbsr_fill(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                   const int32_t *blcPtr, int32_t *outCol, double *outVal, uint16_t *map);
int32_t orc_dbsr_balance(int32_t brow, const int32_t *blcPtr, int32_t *prefix, int32_t cap_prefix,
                         int32_t *overflow);

/* BCSR csrToBcsr (utils/utils.hpp:10-123): pass 1 (bRowPtr NULL) returns
 * nonzeroBlocks; pass 2 fills bRowPtr[rowRegions+1], bColIdx, bVal
 * (tm x tk row-major) and, if non-NULL, the dense mapping. */
int64_t orc_csr2bcsr(int32_t rows, int32_t cols, const int32_t *rowPtr, const int32_t *colIdx, const double *val,
                     int32_t tm, int32_t tk, int32_t *bRowPtr, int32_t *bColIdx, double *bVal, int32_t *mapping);

/* DASP packing (spmv_all, src/dasp.cu:827-1482, rowloop = 1).  Arrays are
 * malloc'd; release with orc_dasp_free. */
typedef struct {
  int32_t row_long, row_block, row_zero, short_row_1, short_row_2, short_row_3, short_row_4;
  int32_t common_13, short_row_34, fill0_nnz_short13, fill0_nnz_short34, fill0_nnz_short;
  int32_t fill0_nnz_long, blocknum, fill0_nnz_reg, nnz_irreg;
  int32_t offset_reg, offset_short1, offset_short13, offset_short34, offset_short22, block_num_all;
  double *short_val, *long_val, *reg_val, *irreg_val;
  int32_t *short_cid, *long_cid, *long_ptr_warp, *reg_cid, *block_ptr, *irreg_cid, *irreg_rpt, *order_rid;
} orc_dasp;
void orc_dasp_pack(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, const double *val, double threshold,
                   int32_t block_longest, orc_dasp *out);
void orc_dasp_free(orc_dasp *o);

/* Block statistics of bench/blockinfo.cpp:96-119 (wrapping 32-bit keys). */
void orc_blockinfo(int32_t rows, const int32_t *rowPtr, const int32_t *colIdx, int64_t *blocks,
                   int64_t *blocks_recorder);

/* Per-block power-of-two-scaled FP16 (dtype 2) / BF16 (dtype 3) BSR: the
 * quantized arrays of the library's bsp_bsr_scaled, and their exact FP64
 * values back in row-major blocks (oracle_formats.c). */
int32_t orc_bsr_scale(int64_t nb, int32_t bs, int32_t dtype, const int32_t *blcIdx, const double *blcVal,
                      uint32_t *key, uint16_t *val);
void orc_bsr_unscale(int64_t nb, int32_t bs, int32_t dtype, const uint32_t *key, const uint16_t *val, double *out);

/* Benchmark input generator (oracle_gen.c): the seeded 27-point stencil with
 * `dof` unknowns per node and the seeded uniform vector, bit-identical to the
 * library's generator.  orc_gen_stencil27 returns nnz (arrays may be NULL to
 * count only; rowPtr alone fills the row pointers), or -1 when too large. */
int64_t orc_gen_stencil27(int32_t m, int32_t dof, uint64_t seed, int32_t *rowPtr, int32_t *colIdx, double *val);
void orc_gen_uniform(int64_t n, uint64_t seed, double *x);

#ifdef __cplusplus
}
#endif
#endif
