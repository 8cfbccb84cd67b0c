/*
 * bsp.h — C ABI of libbspmv, a B200-native (sm_100a) SpMV/SpMM library that
 * drops in for the operator surface of jiajun-c/benchsp (include/spmv.h,
 * include/csrspmv.h, include/amgT.h, include/dasp.h, include/smat.h,
 * include/matrixFormat.hpp).
 *
 * Conventions
 *  - Every entry point returns bsp_status; bsp_last_error() gives a message
 *    for the last failure on the calling thread.  Nothing calls exit().
 *  - Matrix/vector arguments are DEVICE pointers unless the name says _host.
 *  - Every call takes an explicit stream (bsp_stream_t is a cudaStream_t;
 *    NULL means the legacy default stream).  The library never calls
 *    cudaSetDevice: it works on the device current on the calling thread.
 *  - Format descriptors mirror the reference's classes field for field; their
 *    arrays live in device memory allocated by the library and are released by
 *    the matching *_free call.
 *  - Indices are int32 (the reference's CSRFormat<double,int32_t>).  Column
 *    indices of every input CSR must be ascending within a row, without
 *    duplicates (the reference's bench drivers sort COO by (row, col) before
 *    building CSR, bench/spmvfp64.cpp:64-78; its converters assume it).
 */
#ifndef BSP_H
#define BSP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *bsp_stream_t;

typedef enum {
  BSP_OK = 0,
  BSP_ERR_INVALID = 1,      /* bad argument or malformed matrix */
  BSP_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  BSP_ERR_ALLOC = 3,        /* device or host allocation failed */
  BSP_ERR_NOT_CONVERGED = 4,/* iterative solver stopped at its limit */
  BSP_ERR_UNSUPPORTED = 5,  /* combination not implemented */
  BSP_ERR_TIMEOUT = 6       /* a bounded device wait gave up */
} bsp_status;

typedef enum {
  BSP_F64 = 0,
  BSP_F32 = 1,
  BSP_F16 = 2,
  BSP_BF16 = 3
} bsp_dtype;

/* Message for the last non-OK status on this thread ("" if none). */
const char *bsp_last_error(void);
/* Library version string. */
const char *bsp_version(void);

/* ---------------------------------------------------------------------- */
/* Utilities (thin, so tests and hosts without a CUDA binding can move data) */
bsp_status bsp_memcpy_d2h(void *dst_host, const void *src_dev, size_t bytes);
bsp_status bsp_memcpy_h2d(void *dst_dev, const void *src_host, size_t bytes);
bsp_status bsp_device_sync(void);
/* Device memory for hosts without their own CUDA binding (cudaMalloc /
 * cudaFree on the current device). */
bsp_status bsp_device_alloc(void **ptr, size_t bytes);
bsp_status bsp_device_free(void *ptr);
/* Measurement utility (no reference counterpart): `count` gathers of `width`
 * bytes (8, or 16..256 read as width/16 lanes x 16 bytes) at pseudo-random
 * width-aligned offsets of the device buffer `buf` (`bytes` long), eight in
 * flight per thread, one full wave of CTAs.  Time it to get the random-gather
 * rate of the memory level the buffer's size selects (L2 when it fits): the
 * ceiling for kernels whose time goes to scattered x or B-row gathers.
 * `sink` is a device word the kernel writes only on an impossible value. */
bsp_status bsp_gather_probe(const void *buf, size_t bytes, int32_t width, int64_t count, uint64_t seed,
                            void *sink, bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* CSR SpMV  y = alpha*A*x + beta*y
 *
 * Replaces spmv_fp64_warpper / spmv_fp64_balance_warpper
 * (reference src/csrspmv.cu:104 and :136, declared include/csrspmv.h:2-3)
 * and MySpmvWithPrefp64 / MySpmvWithPrefp16 (src/spmv.cu:323 and :197,
 * include/spmv.h:2-3).  Those wrappers upload host arrays, run a timed
 * loop and download y; here the arrays are already on the device and the
 * call launches one kernel on `stream`.
 *
 * algo: BSP_CSR_AUTO picks from the row-length statistics; VECTOR uses a
 * power-of-two group of lanes per row; MERGE is the merge-path (nnz+rows
 * split) kernel, which needs a workspace (see bsp_csr_merge_workspace).
 */
typedef enum {
  BSP_CSR_AUTO = 0,
  BSP_CSR_VECTOR = 1,
  BSP_CSR_MERGE = 2,
  BSP_CSR_SCALAR = 3, /* one thread per row, summing left to right */
  /* a warp per 32 consecutive rows: their nonzero range loaded coalesced in
   * 256-entry pieces, all x gathers of a piece in flight at once, products
   * through shared memory, each row summed left to right by its lane with
   * separately rounded multiply and add (the same results as SCALAR) */
  BSP_CSR_STREAM = 4
} bsp_csr_algo;

/* Values, x and y all have `dtype` storage; F64 accumulates in FP64, the
 * others in FP32.  For F16/BF16 the result is rounded once to the storage
 * type, like ref_spmv_fp16 (src/ref.cpp:3-13).  lanes_per_row: 0 = auto,
 * else 1..32 (power of two) for VECTOR. */
bsp_status bsp_csr_spmv(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *rowPtr, const int32_t *colIdx,
                        const void *values, bsp_dtype dtype, const void *x,
                        void *y, double alpha, double beta, int32_t algo,
                        int32_t lanes_per_row, bsp_stream_t stream);

/* Workspace bytes the merge-path kernel needs for (rows, nnz). */
size_t bsp_csr_merge_workspace(int32_t rows, int32_t nnz);
/* FP64 merge-path SpMV with a caller-provided workspace of at least
 * bsp_csr_merge_workspace(rows, nnz) bytes (16-byte aligned). */
bsp_status bsp_csr_spmv_merge_f64(int32_t rows, int32_t cols, int32_t nnz,
                                  const int32_t *rowPtr, const int32_t *colIdx,
                                  const double *values, const double *x,
                                  double *y, double alpha, double beta,
                                  void *workspace, size_t workspace_bytes,
                                  bsp_stream_t stream);

/* Allocation-free form of bsp_csr_spmv_merge_f64, for callers that may not
 * allocate device memory once they are running (a host that gives all GPU
 * memory to its own pool at start-up, or a latency-critical loop that must
 * not call cudaMalloc/cudaFree, which can synchronize the device).  It has no
 * counterpart in the reference.  The merge-path workspace is a fixed 3 MiB
 * array inside the library, present on every GPU that loads it until the
 * process exits, so rows + nnz must be at most 67,108,864; larger inputs are
 * rejected with BSP_ERR_INVALID.  The array's device address is looked up on
 * the first call on each device (make that first call before any stream
 * capture).  With CUDA's lazy module loading (the default) the array may only
 * be placed in device memory at that first call, so a host that hands its
 * GPU memory to its own pool should make one call per device at start-up,
 * before taking the pool.  All calls share the one array: calls that overlap on the GPU
 * (concurrent streams, threads) race and must be serialized by the caller.
 * Results match bsp_csr_spmv_merge_f64. */
bsp_status bsp_csr_spmv_merge_f64_noalloc(int32_t rows, int32_t cols, int32_t nnz,
                                          const int32_t *rowPtr, const int32_t *colIdx,
                                          const double *values, const double *x,
                                          double *y, double alpha, double beta,
                                          bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* AmgT-style BSR (bsrMAT, reference include/matrixFormat.hpp:59-83).
 * bs = 4 reproduces the reference format exactly; bs = 8 is the same layout
 * with 8x8 blocks (blcMap then holds uint64 bitmaps, bit r*8+c). */
typedef struct {
  int32_t row, col, nnz; /* nnz = blc_num*bs*bs, as CSR2BSR_GPU sets it */
  int32_t blc_row, blc_col, blc_num;
  double stand;   /* std-dev of blocks per block-row (amgT.cu:1146-1155) */
  double avg_nnz; /* true nnz / blc_num (amgT.cu:1136) */
  int32_t *blcPtr;  /* [blc_row+1] */
  int32_t *blcIdx;  /* [blc_num], ascending within a block-row */
  double *blcVal;   /* [blc_num*bs*bs], row-major blocks */
  void *blcMap;     /* [blc_num+1] uint16 (bs=4) or uint64 (bs=8) */
  int32_t warpnum;       /* chunks of <= 64 blocks (common.h:7) */
  int32_t *rowPtrbyWarp; /* [blc_row+1] */
  int32_t *rowIdxbyWarp; /* [warpnum] */
  int32_t bs;
  int32_t true_nnz;
  int32_t dense_blocks; /* blocks whose bitmap is full */
} bsp_bsr;

/* CSR -> BSR on the device; replaces CSR2BSR_GPU + BSR_BALANCED_PREPROCESS_GPU
 * (reference src/amgT.cu:1114 and :1174).  Output arrays are bit-identical to
 * the reference's for bs = 4. */
bsp_status bsp_csr2bsr(int32_t rows, int32_t cols, int32_t nnz,
                       const int32_t *rowPtr, const int32_t *colIdx,
                       const double *values, int32_t bs, bsp_bsr *out,
                       bsp_stream_t stream);
bsp_status bsp_bsr_free(bsp_bsr *m);

typedef enum {
  BSP_BSR_AUTO = 0,
  BSP_BSR_FFMA = 1, /* CUDA-core FP64 FMA, one 256-bit load per block row */
  BSP_BSR_DMMA = 2, /* FP64 mma.sync m8n8k4 on block pairs (4x4 only) */
  BSP_BSR_ADAPTIVE = 3 /* the reference's rule (amgT.cu:1394): DMMA when the
                          average block holds >= 10 nonzeros, FFMA otherwise */
} bsp_bsr_algo;

/* y = alpha*A*x + beta*y for a BSR matrix; replaces the kernels dispatched by
 * amgT_spmv_fp64 (reference src/amgT.cu:1355-1488).  Deterministic: no
 * atomics, every y element written exactly once. */
bsp_status bsp_bsr_spmv(const bsp_bsr *m, const double *x, double *y,
                        double alpha, double beta, int32_t algo,
                        bsp_stream_t stream);

/* FFMA BSR SpMV with an explicit kernel shape (used by the autotuner):
 * lanes_per_blockrow in {4,8,16,32} (bs=4) or {16,32} (bs=8), unroll in
 * {1,2,4} block steps whose loads are issued together, l2_prefetch = 1 adds
 * the 256-byte L2 fetch hint to the value stream.  Shapes without a
 * compiled kernel return BSP_ERR_UNSUPPORTED. */
bsp_status bsp_bsr_spmv_variant(const bsp_bsr *m, const double *x, double *y,
                                double alpha, double beta, int32_t lanes_per_blockrow,
                                int32_t unroll, int32_t l2_prefetch,
                                bsp_stream_t stream);

/* Host-buffer form, the shape of the reference's wrappers (amgT_spmv_fp64,
 * src/amgT.cu:1355, takes host x/y): copies x_host (col doubles) to the
 * device, runs bsp_bsr_spmv, copies y back to y_host (row doubles) and waits
 * for `stream`.  Pinned host buffers give full-bandwidth copies.  beta != 0
 * also uploads y_host first. */
bsp_status bsp_bsr_spmv_host(const bsp_bsr *m, const double *x_host, double *y_host,
                             double alpha, double beta, int32_t algo,
                             bsp_stream_t stream);

/* Host-buffer form with the copies overlapped (no reference counterpart).
 * The plan cuts the block rows into `chunks` ranges (1..64) and keeps device
 * x / y and three streams: x goes up in pieces, each range starts once the x
 * it reads has arrived (its largest column, found at plan time), and its y
 * goes down as soon as it is done.  Pays for matrices whose columns follow
 * their rows (stencils, banded, reordered).  Host buffers should be pinned.
 * The call returns when y_host is written.  The plan records the copies and
 * launches as a CUDA graph for the (x_host, y_host, alpha, beta) it is given
 * and replays that graph while the four repeat, without looking at the
 * buffers again: `m`, its arrays and both host buffers must stay allocated,
 * at their sizes, as long as the plan may be called with those pointers
 * (free `m` only after bsp_bsr_host_plan_destroy). */
typedef struct bsp_bsr_host_plan_s *bsp_bsr_host_plan;
bsp_status bsp_bsr_host_plan_create(const bsp_bsr *m, int32_t chunks,
                                    bsp_bsr_host_plan *plan, bsp_stream_t stream);
bsp_status bsp_bsr_spmv_host_pipelined(bsp_bsr_host_plan plan, const double *x_host,
                                       double *y_host, double alpha, double beta,
                                       bsp_stream_t stream);
/* 1 (default): record the sequence once as a CUDA graph and replay it;
 * 0: issue the copies and launches on the streams at every call. */
bsp_status bsp_bsr_host_plan_set_graph(bsp_bsr_host_plan plan, int32_t use_graph);
/* Caps the grid of each range's SpMV at max_ctas CTAs; 0 = the kernel's own
 * grid.  The plan starts at one wave (8 CTAs per SM; the kernel strides
 * over its block rows), which measured about 2% faster per call than the
 * kernel's own grid on the 27-point stencil. */
bsp_status bsp_bsr_host_plan_set_ctas(bsp_bsr_host_plan plan, int32_t max_ctas);
bsp_status bsp_bsr_host_plan_destroy(bsp_bsr_host_plan plan);

/* ---------------------------------------------------------------------- */
/* BSR with FP16/BF16 values and one power-of-two scale per block.  No
 * reference counterpart: the reference's BSR (bsrMAT, include/matrixFormat.hpp
 * :59-83; SpMV bsr_spmv_tc_fp64, src/amgT.cu:210-274) stores FP64 values
 * only, and its FP16 CSR path (src/spmv.cu:13-27) has no scales.  A block
 * holds bs*bs 16-bit values q and one exponent e; its entries are q * 2^e.
 * e makes the block's largest magnitude land in [2^14, 2^15) for FP16 (the
 * whole normal range below it stays normal) and in [1, 2) for BF16, clamped
 * to [-126, 127]; q = round-to-nearest-even of (float)(a * 2^-e).  Storage per
 * 4x4 block: 32 bytes of values + 4 bytes of key, against 132 for FP64.
 * blcVal is laid out in 4x4 tiles, row-major inside a tile; an 8x8 block is
 * its tiles (0,0), (0,1), (1,0), (1,1) in that order, so every tile is one
 * 32-byte load. */
typedef struct {
  int32_t row, col, bs;          /* bs = 4 or 8 */
  int32_t blc_row, blc_col, blc_num;
  int32_t dtype;                 /* BSP_F16 or BSP_BF16 */
  int32_t *blcPtr;               /* [blc_row+1], as the source BSR */
  uint32_t *blcKey;              /* [blc_num]: block column (bits 0-23) | (e + 128) << 24 */
  uint16_t *blcVal;              /* [blc_num*bs*bs], 4x4 tiles */
} bsp_bsr_scaled;

/* Builds the scaled copy of a BSR matrix on the device (the source is left
 * unchanged and may be freed afterwards).  Needs blc_col < 2^24; values whose
 * block would overflow the target type return BSP_ERR_INVALID. */
bsp_status bsp_bsr_scaled_create(const bsp_bsr *src, int32_t dtype, bsp_bsr_scaled *out,
                                 bsp_stream_t stream);
bsp_status bsp_bsr_scaled_free(bsp_bsr_scaled *m);

/* y = alpha*A*x + beta*y with the scaled matrix: products and sums in FP32
 * (x rounded to FP32 and multiplied by the block's 2^e, which is exact), then
 * alpha*sum + beta*y in the type of y.  x_dtype, y_dtype: BSP_F64 or BSP_F32.
 * Deterministic: every y element is written once, in a fixed order. */
bsp_status bsp_bsr_scaled_spmv(const bsp_bsr_scaled *m, const void *x, int32_t x_dtype, void *y,
                               int32_t y_dtype, double alpha, double beta, bsp_stream_t stream);

/* The same with an explicit lane count per block row (4, 8, 16 or 32; for
 * bs = 8 at least 4) and 1 or 2 blocks per lane per loop trip (tuning). */
bsp_status bsp_bsr_scaled_spmv_variant(const bsp_bsr_scaled *m, const void *x, int32_t x_dtype,
                                       void *y, int32_t y_dtype, double alpha, double beta,
                                       int32_t lanes_per_blockrow, int32_t unroll,
                                       bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Fixed-tile BCSR (BCSRFormat<double,int32_t>, reference
 * include/matrixFormat.hpp:16-30).  blockNum is 64-bit (rowRegions *
 * colRegions overflows int32 for n above ~46k with 1x1 tiles). */
typedef struct {
  int32_t *bcsrRowPtr;                /* [rowRegions+1] */
  int32_t *bcsrcolIdx;                /* [nonzeroBlocks] block columns, ascending */
  int32_t *relativeBlockIndexMapping; /* [rowRegions*colRegions], -1 = empty; NULL unless requested */
  double *values;                     /* [nonzeroBlocks*TILE_M*TILE_K] row-major tiles */
  int32_t row, col;
  int64_t blockNum;                   /* rowRegions * colRegions */
  int32_t TILE_M, TILE_N, TILE_K;     /* TILE_N = TILE_K */
  int32_t nnz;                        /* nonzeros of the source CSR */
  int32_t colRegions, rowRegions, nonzeroBlocks, elemCount;
  int32_t block_row, block_col;       /* = rowRegions, colRegions */
} bsp_bcsr;

/* CSR -> BCSR with tile_m x tile_k tiles (1..64 each) on the device;
 * replaces csrToBcsr (reference utils/utils.hpp:10), whose dense
 * rowRegions x colRegions table limits it to small matrices.  Arrays are
 * bit-identical to the reference's; with_mapping = 1 also builds the dense
 * relativeBlockIndexMapping. */
bsp_status bsp_csr2bcsr(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *rowPtr, const int32_t *colIdx,
                        const double *values, int32_t tile_m, int32_t tile_k,
                        int32_t with_mapping, bsp_bcsr *out, bsp_stream_t stream);
bsp_status bsp_bcsr_free(bsp_bcsr *b);
/* y = alpha*A*x + beta*y for any tile shape; replaces bcsr_spmv_fp64
 * (reference src/bcsr.cu:224, include/bcsr.h:3). */
bsp_status bsp_bcsr_spmv(const bsp_bcsr *b, const double *x, double *y,
                         double alpha, double beta, bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* DBSR, "denser" 4x4 blocks (dbsrMat, reference include/matrixFormat.hpp:86-106).
 * The z-th nonzero of row i sits in block blcPtr[i/4] + z/4 at position
 * (i%4)*4 + z%4, with its own column index (padding: column 0, value 0). */
typedef struct {
  int32_t row, col, nnz;
  int32_t blc_row, blc_col, blc_num; /* blc_num = blocks (blocknnz / 16) */
  double stand, avg_nnz;
  int32_t *blcPtr;      /* [blc_row+1] */
  int32_t *colIdx;      /* [blocknnz] per-element column indices */
  double *blcVal;       /* [blocknnz] */
  uint16_t *blcMap;     /* [blc_num] (+ padding to whole 32-bit words) */
  int32_t blocknnz;     /* blc_num * 16 */
  int32_t warpnum;      /* warps of <= 64 blocks from balanceDbsr */
  int32_t *rowPtrbyWarp;/* unused (NULL), kept for the field layout */
  int32_t *rowIdxbyWarp;/* unused (NULL) */
  int32_t *recorderMap; /* [row] new -> old row (recorder variant), else NULL */
  int32_t *prefix;      /* [warpnum+1] balanceDbsr warp -> block-row prefix */
  int32_t balance_overflow; /* 1 where the reference's balanceDbsr would index
                               past its warp vector (see bsp_csr2dbsr) */
} bsp_dbsr;

/* CSR -> DBSR on the device, bit-identical to the reference's host
 * converters: recorder = 0 replaces csrTodbsr + balanceDbsr
 * (include/dbsr.h:10 and :94); recorder = 1 replaces csrTodbsrWithRecorder
 * (include/dbsr.h:208: rows sorted ascending by length, ties by index).
 * balanceDbsr's second walk can run past the warp count of its first walk
 * (the reference then writes out of bounds); the walk is replayed exactly,
 * the warp list grows to hold it and balance_overflow is set. */
bsp_status bsp_csr2dbsr(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *rowPtr, const int32_t *colIdx,
                        const double *values, int32_t recorder, bsp_dbsr *out,
                        bsp_stream_t stream);
bsp_status bsp_dbsr_free(bsp_dbsr *m);
/* y = alpha*A*x + beta*y; replaces amgT_spmv_fp64_dbsr(_balance)
 * (reference src/amgT.cu:1202, :1280; include/amgT.h:4-5), whose kernels
 * compute row sums (they overwrite the gathered x with 1.0, amgT.cu:356,
 * :425) -- this one computes A*x.  permuted_output = 1 writes y in the
 * recorder order (the reference's layout, un-permuted by its caller,
 * bench/spmvfp64.cpp:162-166); 0 writes y in the original row order. */
bsp_status bsp_dbsr_spmv(const bsp_dbsr *m, const double *x, double *y,
                         double alpha, double beta, int32_t permuted_output,
                         bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* DASP packing (the arrays spmv_all builds and uploads, reference
 * src/dasp.cu:814-1600).  Row classes: len 1, 2, 3, 4, 0, long
 * (>= block_longest) and row-block rows.  y slots run in order_rid order:
 * long rows, row-block rows (sorted descending by length), len-1 rows,
 * 1&3 tile pairs (8 len-1 then 8 len-3 rows per tile), remaining len-3,
 * len-4, len-2 rows, empty rows. */
typedef struct {
  int32_t rows, cols, nnz;
  double threshold;
  int32_t block_longest;
  int32_t row_long, row_block, row_zero;
  int32_t short_row_1, short_row_2, short_row_3, short_row_4; /* _1/_3 after pairing */
  int32_t common_13, short_row_34;
  int32_t short_block13, short_block34, short_block22;
  int32_t blocknum;       /* 8-row blocks, padded to a multiple of 4 */
  int32_t long_warps;     /* 64-value chunks of the long rows */
  int32_t warp_number;    /* long_warps padded to a multiple of 4 */
  int32_t fill0_nnz_long, fill0_nnz_short13, fill0_nnz_short34, fill0_nnz_short22;
  int32_t fill0_nnz_short, fill0_nnz_reg, nnz_irreg;
  /* the reference kernel's block ranges (dasp.cu:1531-1539) */
  int32_t offset_reg, offset_short1, offset_short13, offset_short34, offset_short22, block_num_all;
  double *long_val;  int32_t *long_cid;        /* [fill0_nnz_long] */
  int32_t *long_ptr_warp;                      /* [row_long+1] chunk prefix */
  int32_t *long_row_of_warp;                   /* [warp_number], -1 = padding */
  double *warp_val;  int32_t *long_done;       /* SpMV scratch: chunk partials, arrival counters */
  double *reg_val;   int32_t *reg_cid;         /* [fill0_nnz_reg] 8x4 tiles */
  int32_t *block_ptr;                          /* [blocknum+1] */
  double *irreg_val; int32_t *irreg_cid;       /* [nnz_irreg] */
  int32_t *irreg_rpt;                          /* [row_block+1] */
  double *short_val; int32_t *short_cid;       /* [fill0_nnz_short] */
  int32_t *order_rid;                          /* [rows] y slot -> row */
  int32_t *sorted_rid;                         /* [row_block] row-block rows, sorted */
  int32_t *row_len_sorted;                     /* [row_block+1] prefix of their lengths */
  /* SpMV work split of the long rows: groups of up to 8 consecutive chunks
   * of one row, one warp each */
  int32_t long_groups;
  int32_t *long_group_ptr;                     /* [row_long+1] group prefix */
  int32_t *long_group_info;                    /* [4*long_groups] per group: long-row
                                                  index, first chunk, first group of
                                                  the row, chunks | row's groups << 4 */
} bsp_dasp;

/* CSR -> DASP on the device, arrays bit-identical to spmv_all's host
 * packing (reference src/dasp.cu:827-1482) for the same threshold and
 * block_longest (the reference bench passes 0.75 and 256,
 * bench/spmvfp64.cpp:177).  threshold must be > 0 (the reference loops
 * forever on an empty block otherwise). */
bsp_status bsp_csr2dasp(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *rowPtr, const int32_t *colIdx,
                        const double *values, double threshold,
                        int32_t block_longest, bsp_dasp *out, bsp_stream_t stream);
bsp_status bsp_dasp_free(bsp_dasp *d);
/* y = alpha*A*x + beta*y in one launch (the reference needs dasp_spmv2 +
 * longPart_sum, dasp.cu:406, :381).  permuted_output = 1 writes y in
 * order_rid order, as spmv_all returns it; 0 writes the original row order.
 * Calls on one bsp_dasp must not overlap on the GPU (they share the
 * long-row scratch). */
bsp_status bsp_dasp_spmv(const bsp_dasp *d, const double *x, double *y,
                         double alpha, double beta, int32_t permuted_output,
                         bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* SpMM C = alpha*A*B + beta*C (B: cols x N, C: rows x N, both row-major;
 * C is FP32).  Replaces smatSpmmfp16 (reference src/smat.cu:103,
 * include/smat.h:1), whose kernel accumulates in FP16 and never writes its
 * output; here the accumulation is FP32.
 *
 * CSR form: values and B share `dtype` (F16, BF16 or F32), any sparsity.
 * Outside stream capture the call first reads back the longest row length
 * (one small kernel; it waits for the stream); when a row exceeds 8192
 * nonzeros and 64x the mean, a temporary row-split plan (below) is built,
 * used and freed.  Callers that repeat the product on such a matrix should
 * keep their own plan (bsp_spmm_plan_create + bsp_spmm_csr_planned). */
bsp_status bsp_spmm_csr(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *rowPtr, const int32_t *colIdx,
                        const void *values, bsp_dtype dtype, const void *B,
                        int32_t N, int64_t ldb, float *C, int64_t ldc,
                        float alpha, float beta, bsp_stream_t stream);

/* Row-split CSR form for power-law rows: the plan cuts rows longer than
 * `chunk` nonzeros into chunks processed by separate warps; their partial
 * rows go to a workspace of bsp_spmm_plan_workspace(plan, N) bytes and are
 * summed in a fixed order (deterministic): groups of up to 32 consecutive
 * chunks by separate warps, then each row's group sums.
 *
 * Two engines run a planned product.  "grouped": one warp per row or chunk
 * over all N columns in one pass.  "slab": the columns are taken in slabs of
 * up to 32 lanes x 16 bytes of B row (256 FP16 columns; one pass over A per
 * slab), rows of at most `chunk` nonzeros, sorted by length, are spread one
 * per group of lanes (several rows per warp in flight), and long-row chunks
 * keep a warp each.  The default is the slab engine whenever B's rows are
 * 16-byte aligned and N is a multiple of 16 bytes of elements.  The engines
 * sum in different orders: results differ in rounding, each within the FP32
 * accumulation bound. */
typedef struct {
  int32_t rows, chunk;
  int64_t nchunks, nparts;
  int32_t nsplit;
  int32_t *chunk_ptr;  /* [rows+1] */
  int32_t *part_ptr;   /* [rows+1] partial-row slots of split rows */
  int32_t *chunk_row;  /* [nchunks] */
  int32_t *split_rows; /* [nsplit] */
  int32_t nshort;      /* rows of at most `chunk` nonzeros (empty rows included) */
  int32_t *short_rows; /* [nshort] those rows, longest first (stable) */
  int32_t *long_chunk; /* [nparts] chunk index of each partial-row slot */
  int32_t *long_se;    /* [2*nparts] (start, end) nonzero range of each slot's chunk */
  int32_t *short_se;   /* [2*nshort] (start, end) nonzero range of each listed short row */
  int32_t slab_l2_hints; /* slab engine cache policy for slabs of B of at most 64 MiB
                            (cols x slab width; wider slabs use default caching), set to
                            1 by bsp_spmm_plan_create: 1 = A's entries loaded and C
                            stored as evict-first, the gathered B slab rows as
                            evict-last, so the slab stays in L2 for the pass; 2 = A and
                            C evict-first, B default; 0 = default caching */
  int32_t ngroups;       /* groups of up to 32 consecutive chunks of the split rows */
  int32_t *group_ptr;    /* [nsplit+1] first group of each split row */
  int32_t *group_split;  /* [ngroups] split-row index of each group */
} bsp_spmm_plan;

bsp_status bsp_spmm_plan_create(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                int32_t chunk, bsp_spmm_plan *plan,
                                bsp_stream_t stream);
bsp_status bsp_spmm_plan_free(bsp_spmm_plan *plan);
size_t bsp_spmm_plan_workspace(const bsp_spmm_plan *plan, int32_t N);
bsp_status bsp_spmm_csr_planned(const bsp_spmm_plan *plan, int32_t cols, int32_t nnz,
                                const int32_t *rowPtr, const int32_t *colIdx,
                                const void *values, bsp_dtype dtype, const void *B,
                                int32_t N, int64_t ldb, float *C, int64_t ldc,
                                float alpha, float beta, void *workspace,
                                size_t workspace_bytes, bsp_stream_t stream);

typedef enum { BSP_SPMM_AUTO = 0, BSP_SPMM_GROUPED = 1, BSP_SPMM_SLAB = 2 } bsp_spmm_engine;

/* bsp_spmm_csr_planned with the engine and, for the slab engine, the slab
 * width (columns per pass; 0 = the default; otherwise 1..32 lanes, a power
 * of two, times 16 bytes of B row, dividing N) chosen by the caller. */
bsp_status bsp_spmm_csr_planned_variant(const bsp_spmm_plan *plan, int32_t cols, int32_t nnz,
                                        const int32_t *rowPtr, const int32_t *colIdx,
                                        const void *values, bsp_dtype dtype, const void *B,
                                        int32_t N, int64_t ldb, float *C, int64_t ldc,
                                        float alpha, float beta, void *workspace,
                                        size_t workspace_bytes, int32_t engine,
                                        int32_t slab_cols, bsp_stream_t stream);

/* Block (SMaT) form: 16x16 tiles of the matrix (the reference's csrToBcsr
 * with TILE_M = TILE_K = 16, smat.cu:116-120) in F16 or BF16, staged with
 * bulk asynchronous copies and multiplied with tensor-core MMA (FP32
 * accumulation).  Pays when tiles are dense (`fill` = nnz / stored tile
 * entries). */
typedef struct {
  int32_t rows, cols, nnz;
  int32_t dtype;      /* BSP_F16 or BSP_BF16 */
  bsp_bcsr tiles;     /* 16x16 structure (tiles.values released) */
  void *tile_val;     /* [tiles.nonzeroBlocks*256] F16/BF16 tiles, each as four
                         8x8 core matrices (tcgen05 K-major operand order) */
  int32_t *err;       /* device flag: a bounded wait timed out */
  double fill;
} bsp_smat;

bsp_status bsp_smat_create(int32_t rows, int32_t cols, int32_t nnz,
                           const int32_t *rowPtr, const int32_t *colIdx,
                           const double *values, bsp_dtype dtype, bsp_smat *out,
                           bsp_stream_t stream);
bsp_status bsp_smat_free(bsp_smat *m);
/* B: dtype of the matrix, 16-byte aligned, ldb % 8 == 0; N % 32 == 0.
 * Runs on the tcgen05 tensor cores (TMEM accumulators, TMA staging of B):
 * resident CTAs walk every (block row, slab of 128 C columns, or 64 when
 * N < 128); bsp_smat_spmm_path can ask for the other kernels. */
bsp_status bsp_smat_spmm(const bsp_smat *m, const void *B, int32_t N,
                         int64_t ldb, float *C, int64_t ldc, float alpha,
                         float beta, bsp_stream_t stream);
typedef enum {
  BSP_SMAT_AUTO = 0,
  BSP_SMAT_MMA_SYNC = 1, /* warp mma.sync.m16n8k16, FP32 accumulators in registers */
  BSP_SMAT_TCGEN05 = 2,  /* tcgen05.mma M=128 N=16 K=16 per tile: the persistent kernel (5) */
  BSP_SMAT_TCGEN05_W64 = 3,  /* tcgen05, one CTA per block row, 64 C columns per CTA */
  BSP_SMAT_TCGEN05_W128 = 4, /* tcgen05, one CTA per block row, 128 C columns per CTA */
  BSP_SMAT_TCGEN05_PERSISTENT = 5, /* tcgen05, resident CTAs walking every block row: a producer
                                     warp, an MMA warp and four epilogue warps, two TMEM
                                     accumulators so one block row's read-out overlaps the
                                     next one's MMAs */
  BSP_SMAT_TCGEN05_PERSISTENT_W64 = 6 /* the persistent form in 64-column slabs */
} bsp_smat_path;
bsp_status bsp_smat_spmm_path(const bsp_smat *m, const void *B, int32_t N,
                              int64_t ldb, float *C, int64_t ldc, float alpha,
                              float beta, int32_t path, bsp_stream_t stream);
/* Reads the device error flag (waits for `stream`): BSP_ERR_TIMEOUT when a
 * bounded copy wait gave up. */
bsp_status bsp_smat_check(const bsp_smat *m, bsp_stream_t stream);

/* Gathered-tile form of the SMaT SpMM for matrices whose nonzeros scatter
 * over all columns (graph adjacency), where 16x16 tiles of the matrix as
 * given hold a handful of entries (the 2^20-row power-law graph: 14.9M
 * tiles, 0.8% full, 7.6 GB in FP16, more than int32 tile indexing holds).
 * Each group of 16 rows keeps its distinct columns in chunks of 16 and the
 * 16x16 tile of its values in those columns; the product gathers a chunk's
 * 16 B rows into shared memory and runs the same tcgen05.mma as the block
 * path (persistent CTAs, two TMEM accumulators).  No reference counterpart
 * (the reference's SMaT, src/smat.cu:22-91, only has the plain tiles).
 * Built on the host from host CSR arrays; FP16 or BF16; N % 8 == 0; groups
 * with more than 64 chunks are split and summed in a fixed order through a
 * workspace of bsp_gtile_workspace(g, N) bytes. */
typedef struct {
  int32_t rows, cols, nnz, dtype;
  int64_t nchunks;
  int32_t ngroups, npieces, nsplit, nslots;
  int32_t *piece_ptr;    /* [npieces+1] chunk ranges */
  int32_t *piece_group;  /* [npieces] */
  int32_t *piece_slot;   /* [npieces] partial-row slot, -1 when the piece is its group's only one */
  int32_t *group_piece;  /* [ngroups+1] piece ranges of each group */
  int32_t *split_groups; /* [nsplit] groups with more than one piece */
  int32_t *chunk_cols;   /* [nchunks*16] gathered B rows (0 in padding slots) */
  void *chunk_tiles;     /* [nchunks*256] FP16/BF16 tiles, tcgen05 K-major core layout */
  int32_t *err;          /* device flag: a bounded wait gave up */
} bsp_gtile;
bsp_status bsp_gtile_create_host(int32_t rows, int32_t cols, int32_t nnz, const int32_t *rowPtr,
                                 const int32_t *colIdx, const double *values, bsp_dtype dtype,
                                 bsp_gtile *out);
size_t bsp_gtile_workspace(const bsp_gtile *g, int32_t N);
bsp_status bsp_gtile_spmm(const bsp_gtile *g, const void *B, int32_t N, int64_t ldb, float *C,
                          int64_t ldc, float alpha, float beta, void *workspace,
                          size_t workspace_bytes, bsp_stream_t stream);
bsp_status bsp_gtile_check(const bsp_gtile *g, bsp_stream_t stream);
bsp_status bsp_gtile_free(bsp_gtile *g);

/* ---------------------------------------------------------------------- */
/* Conjugate gradients (absent in the reference): plain FP64 CG, or
 * mixed-precision CG with reliable updates -- iterations run on the matrix
 * stored in FP32, or FP16/BF16 with one power-of-two exponent per 32
 * nonzeros, with int16 column offsets when every |col - row| < 32768, and
 * FP32 vectors; whenever the iterated residual has dropped by reliable_delta
 * the solution is folded into the FP64 x and the residual is replaced by the
 * FP64 b - A x (search direction kept).  Convergence: ||b - A x|| / ||b|| <=
 * tol, computed in FP64. */
typedef enum {
  BSP_CG_FP64 = 0,
  BSP_CG_MIXED_F32 = 1,
  BSP_CG_MIXED_F16 = 2,
  BSP_CG_MIXED_BF16 = 3
} bsp_cg_mode;

/* Preconditioner (applied in the iteration precision): none; Jacobi (the
 * inverse diagonal); block-Jacobi (the inverses of the diagonal blocks of
 * precond_block consecutive rows, e.g. the dof blocks of a BSR matrix; the last
 * block is padded with identity rows).  create fails with BSP_ERR_INVALID on a
 * zero diagonal entry or a singular block. */
/* How the mixed modes reach the FP64 tolerance.  RELIABLE: one CG on the
 * low-precision matrix whose residual is replaced by the FP64 one (and the
 * solution folded into x64) each time it has dropped by reliable_delta; the
 * search direction is kept, so the count stays that of FP64 CG while the
 * low-precision matrix is close to A.  FLEXIBLE: an FP64 flexible CG (one
 * previous direction, FP64 matrix) whose preconditioner is the low-precision
 * (P)CG run until its residual has dropped by reliable_delta; it keeps
 * converging when the low-precision matrix is far from A (large condition
 * number times storage rounding).  AUTO: RELIABLE, switching to FLEXIBLE when
 * a replaced residual is far above the iterated one. */
typedef enum {
  BSP_CG_REFINE_AUTO = 0,
  BSP_CG_REFINE_RELIABLE = 1,
  BSP_CG_REFINE_FLEXIBLE = 2
} bsp_cg_refine;

typedef enum {
  BSP_CG_PRECOND_NONE = 0,
  BSP_CG_PRECOND_JACOBI = 1,
  BSP_CG_PRECOND_BLOCK_JACOBI = 2
} bsp_cg_precond;

typedef struct {
  int32_t mode;          /* bsp_cg_mode */
  double tol;            /* relative residual target (1e-10) */
  int32_t max_iters;     /* CG iteration budget */
  int32_t check_every;   /* iterations per CUDA graph between host checks (rounded up to even) */
  double reliable_delta; /* mixed modes: residual drop that triggers an FP64 update (0.1) */
  int32_t use_graphs;    /* 1: replay captured iteration chunks */
  int32_t precond;       /* bsp_cg_precond */
  int32_t precond_block; /* BLOCK_JACOBI: rows per diagonal block, 4 or 8 */
  int32_t refine;        /* bsp_cg_refine (mixed modes) */
} bsp_cg_options;

typedef struct {
  int32_t iterations;       /* CG iterations */
  int32_t reliable_updates; /* FP64 residual replacements */
  double rel_residual;      /* final ||b - A x|| / ||b|| in FP64 */
  double seconds;           /* device time of the solve (CUDA events) */
  int32_t converged;
  int64_t bytes_moved;      /* algorithmic bytes of all kernels */
  int32_t delta16;          /* int16 column offsets were used */
  int32_t outer_steps;      /* mixed modes: outer flexible steps taken (0 when
                               residual replacement sufficed) */
} bsp_cg_result;

typedef struct bsp_cg_plan_s *bsp_cg_plan;

bsp_status bsp_cg_default_options(bsp_cg_options *opt);
/* Prepares a solver for the SPD CSR matrix (device arrays, kept by
 * reference: they must outlive the plan): the low-precision copy, vectors,
 * and (on first solve) the captured iteration graphs. */
bsp_status bsp_cg_create(int32_t n, int32_t nnz, const int32_t *rowPtr,
                         const int32_t *colIdx, const double *values,
                         const bsp_cg_options *opt, bsp_cg_plan *plan,
                         bsp_stream_t stream);
/* Solves A x = b; x holds the initial guess on entry.  Returns
 * BSP_ERR_NOT_CONVERGED (with res filled) when tol is not reached. */
bsp_status bsp_cg_solve(bsp_cg_plan plan, const double *b, double *x,
                        bsp_cg_result *res, bsp_stream_t stream);
bsp_status bsp_cg_destroy(bsp_cg_plan plan);
/* k right-hand sides at once: A X = B with B, X device arrays, row-major with
 * leading dimensions ldb, ldx >= k (row i, column j at B[i*ldb + j]); X holds
 * the initial guesses on entry.  Every column runs its own FP64 CG (same
 * iterates as k separate solves) but each iteration reads the matrix once
 * for up to 8 columns.  Needs a plan with mode BSP_CG_FP64 and precond NONE
 * or JACOBI (else BSP_ERR_UNSUPPORTED).  rel_residuals (k entries, may be
 * NULL) receives each column's final ||b - A x|| / ||b||; res aggregates
 * (iterations = the most any column group ran, rel_residual = the worst).
 * BSP_ERR_NOT_CONVERGED when a column stops above the tolerance. */
bsp_status bsp_cg_solve_multi(bsp_cg_plan plan, int32_t k, const double *B,
                              int64_t ldb, double *X, int64_t ldx,
                              double *rel_residuals, bsp_cg_result *res,
                              bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* 4x4 block statistics of bench/blockinfo.cpp:96-119 (reference): the number
 * of distinct 4x4 blocks of the matrix (keys row/4*1000005 + col/4) and of
 * its DBSR-style packing (keys row/4*1000005 + z/4, z = position in the row),
 * counted on wrapped 32-bit keys exactly as the reference's int arithmetic
 * does.  Average nonzeros per block = nnz / count. */
bsp_status bsp_blockinfo(int32_t rows, int32_t cols, int32_t nnz,
                         const int32_t *rowPtr, const int32_t *colIdx,
                         int64_t *blocks, int64_t *blocks_recorder,
                         bsp_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Reordering (no reference counterpart; the reference blocks matrices in the
 * order given, src/smat.cu:116-120).  Reverse Cuthill-McKee on the pattern
 * of A + A^T: perm[new] = old.  Gathers nonzeros near the diagonal, which
 * raises BSR block and SMaT tile fill for matrices numbered without
 * locality.  Runs on the host (a one-time preprocessing step); the device
 * forms copy in and out and wait for `stream`. */
bsp_status bsp_reorder_rcm(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                           const int32_t *colIdx, int32_t *perm,
                           bsp_stream_t stream);
/* P A P^T of a square CSR matrix (new row i = old row perm[i], columns
 * renumbered and sorted); values may be NULL (pattern only). */
bsp_status bsp_permute_csr(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                           const int32_t *colIdx, const double *values,
                           const int32_t *perm, int32_t *outRowPtr,
                           int32_t *outColIdx, double *outValues,
                           bsp_stream_t stream);
/* The same on host arrays. */
bsp_status bsp_reorder_rcm_host(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                const int32_t *colIdx, int32_t *perm);
bsp_status bsp_permute_csr_host(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                const int32_t *colIdx, const double *values,
                                const int32_t *perm, int32_t *outRowPtr,
                                int32_t *outColIdx, double *outValues);
/* Row-similarity order for tile formats (SMaT 16x16 tiles, BSR blocks): rows
 * whose nonzeros fall in the same `block_cols`-wide column blocks are put in
 * the same group of `group_rows` consecutive rows; perm[new] = old.  Rows are
 * grouped greedily by the Jaccard similarity of their column-block sets
 * (seeds in row order, candidates from an inverted index with bounded
 * scans, ties by row index; empty rows last), so it is deterministic.  For
 * rectangular matrices too: apply it with bsp_permute_rows_csr (P A) and
 * read row i of the product as original row perm[i].  Host code; the device
 * form copies in and out and waits for `stream`. */
bsp_status bsp_reorder_similarity(int32_t rows, int32_t cols, int32_t nnz,
                                  const int32_t *rowPtr, const int32_t *colIdx,
                                  int32_t group_rows, int32_t block_cols,
                                  int32_t *perm, bsp_stream_t stream);
bsp_status bsp_reorder_similarity_host(int32_t rows, int32_t cols, int32_t nnz,
                                       const int32_t *rowPtr, const int32_t *colIdx,
                                       int32_t group_rows, int32_t block_cols,
                                       int32_t *perm);
/* SpMM engine choice for C = A B with N columns of B, sharing the
 * reordering with the SMaT path: counts the 16x16 tiles of A and the chunks
 * of its gathered-tile form (16 distinct columns of a 16-row group) as given
 * and, when `perm` (rows entries) is not NULL, after bsp_reorder_similarity
 * (written to perm), and estimates each engine from B200 measurements
 * (SMaT time per tile, gathered-tile time per chunk, grouped CSR time per
 * nonzero, all per column of B).  engine = BSP_SPMM_ENGINE_SMAT or
 * BSP_SPMM_ENGINE_GTILE (build that matrix from the rows in perm order when
 * reorder = 1, and read row i of C as original row perm[i]; smat_path says
 * which tile path) or BSP_SPMM_ENGINE_CSR (bsp_spmm_csr on A as given).
 * SMaT needs N % 32 == 0, the gathered tiles N % 8 == 0; the estimates are
 * -1 where an engine does not apply.  Host code, a one-time decision per
 * matrix. */
enum { BSP_SPMM_ENGINE_CSR = 0, BSP_SPMM_ENGINE_SMAT = 1, BSP_SPMM_ENGINE_GTILE = 2 };
typedef struct bsp_spmm_choice {
  int32_t engine;
  int32_t smat_path;   /* BSP_SMAT_TCGEN05 */
  int32_t reorder;     /* 1: the chosen matrix is built from the rows in perm order */
  int32_t reserved;
  int64_t tiles_given, tiles_reordered;   /* tiles_reordered = -1 without perm */
  double est_seconds_smat_given, est_seconds_smat_reordered, est_seconds_csr;
  int64_t chunks_given, chunks_reordered; /* chunks_reordered = -1 without perm */
  double est_seconds_gtile_given, est_seconds_gtile_reordered;
} bsp_spmm_choice;
bsp_status bsp_spmm_choose_host(int32_t rows, int32_t cols, int32_t nnz,
                                const int32_t *rowPtr, const int32_t *colIdx,
                                int32_t N, int32_t *perm, bsp_spmm_choice *out);
/* P A, rows only (new row i = old row perm[i], its entries as stored; any
 * column count); values may be NULL (pattern only). */
bsp_status bsp_permute_rows_csr(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                const int32_t *colIdx, const double *values,
                                const int32_t *perm, int32_t *outRowPtr,
                                int32_t *outColIdx, double *outValues,
                                bsp_stream_t stream);
bsp_status bsp_permute_rows_csr_host(int32_t rows, int32_t nnz, const int32_t *rowPtr,
                                     const int32_t *colIdx, const double *values,
                                     const int32_t *perm, int32_t *outRowPtr,
                                     int32_t *outColIdx, double *outValues);

/* ---------------------------------------------------------------------- */
/* Format autotuner for FP64 SpMV (no reference counterpart: the reference's
 * drivers run every format on every matrix, bench/spmvfp64.cpp:135-177).
 * Model mode decides from row-length statistics and exact 4x4 / 8x8 block
 * counts; measure mode converts to each candidate that can pay off, times
 * them and keeps the fastest.  Results are cached per process by a
 * structural hash of (rows, cols, nnz, rowPtr, colIdx); with the environment
 * variable BSP_TUNE_CACHE set to a file path, the cache is also read from
 * and appended to that file. */
typedef enum { BSP_FMT_CSR = 0, BSP_FMT_BSR = 1, BSP_FMT_DASP = 2 } bsp_format;

typedef struct {
  int32_t format;   /* bsp_format */
  int32_t csr_algo; /* BSP_CSR_VECTOR or BSP_CSR_MERGE (format CSR) */
  int32_t lanes;    /* lanes per row (CSR vector) */
  int32_t bs;       /* 4 or 8 (format BSR) */
  int32_t bsr_algo; /* BSP_BSR_FFMA / DMMA / ADAPTIVE (format BSR) */
  int32_t from_cache;
  double spmv_us;   /* measured time of the choice (measure mode), else 0 */
  uint64_t key;     /* structural hash */
  /* statistics the model used */
  double mean_len, cv_len, fill4, fill8;
  int32_t max_len;
  int32_t long_rows; /* rows with >= 256 nonzeros */
} bsp_tune_result;

bsp_status bsp_tune_spmv(int32_t rows, int32_t cols, int32_t nnz,
                         const int32_t *rowPtr, const int32_t *colIdx,
                         const double *values, int32_t measure,
                         bsp_tune_result *out, bsp_stream_t stream);
/* Structural hash only. */
bsp_status bsp_matrix_key(int32_t rows, int32_t cols, int32_t nnz,
                          const int32_t *rowPtr, const int32_t *colIdx,
                          uint64_t *key, bsp_stream_t stream);
void bsp_tune_cache_clear(void);

/* A tuned SpMV executor: holds the chosen format's arrays (the CSR arrays
 * must stay alive for the CSR choice). */
typedef struct bsp_spmv_plan_s *bsp_spmv_plan;
bsp_status bsp_spmv_plan_create(int32_t rows, int32_t cols, int32_t nnz,
                                const int32_t *rowPtr, const int32_t *colIdx,
                                const double *values, int32_t measure,
                                bsp_spmv_plan *plan, bsp_stream_t stream);
bsp_status bsp_spmv_plan_choice(bsp_spmv_plan plan, bsp_tune_result *out);
/* y = alpha*A*x + beta*y in the original row order. */
bsp_status bsp_spmv_plan_run(bsp_spmv_plan plan, const double *x, double *y,
                             double alpha, double beta, bsp_stream_t stream);
bsp_status bsp_spmv_plan_destroy(bsp_spmv_plan plan);

/* ---------------------------------------------------------------------- */
/* Batched SpMV / SpMM over many independent CSR matrices (no reference
 * counterpart: the reference launches one matrix at a time, e.g.
 * src/csrspmv.cu:104-170).  One persistent kernel processes a work list
 * built at plan time: row items (a run of consecutive rows, `lanes` lanes
 * per row, chosen per matrix by the tuner) and long-row segments (rows
 * longer than long_row_nnz, cut into seg_nnz-sized pieces whose partial
 * sums the last-arriving warp adds in segment order).  Results are
 * deterministic.  Warps take items from a counter, long segments first.
 * The launch (counter reset + kernel) is captured once in a CUDA graph.
 * y_m = A_m x_m for every matrix m; with nrhs = 8, x_m and y_m are
 * row-major rows x 8 / cols x 8 blocks.
 *
 * Per matrix the plan also picks the storage: CSR as given, or a SELL-32
 * copy it builds (slices of 32 rows padded to the slice's longest row, entry
 * k of slice row l at slice_start + 32k + l, values in the batch's type),
 * which a warp reads one slice at a time with every access coalesced.
 * Narrow form (the default): the rows in order with 16-bit column offsets
 * from the row, for matrices whose padding adds at most 1/8, with no row
 * longer than long_row_nnz and every |column - row| < 32768.  Wide form
 * (opt-in, sell_wide = 1): the rows of at most T entries sorted by length,
 * 32-bit columns and a row permutation, T the largest power of two at which
 * padding adds at most 1/8, rows above T as whole-warp segments; it measured
 * slower than CSR on power-law rows (512-matrix batch, Zipf half: 534 vs 107
 * us), so it is off by default.  SELL matrices are chosen by these rules;
 * for the CSR ones tune = 1 times the lane counts per matrix. */
typedef struct {
  int32_t rows, cols, nnz;
  const int32_t *rowPtr; /* device */
  const int32_t *colIdx; /* device */
  const void *values;    /* device, F64 or F32 */
  const void *x;         /* device, cols * nrhs */
  void *y;               /* device, rows * nrhs */
} bsp_batch_mat;

typedef struct {
  int32_t tune;         /* 0: row-statistics model, 1: time candidates */
  int32_t seg_nnz;      /* nonzeros per long-row segment (default 512) */
  int32_t long_row_nnz; /* rows above this are split (default 1024) */
  int32_t item_nnz;     /* target nonzeros per row item, 0 = automatic */
  int32_t use_graph;    /* capture the launch in a CUDA graph (default 1) */
  int32_t sell;         /* 1: store qualifying matrices as SELL-32 (default 1) */
  int32_t sell_wide;    /* 1: also the wide (length-sorted) SELL-32 form (default 0) */
} bsp_batch_options;

typedef struct bsp_batch_plan_s *bsp_batch_plan;

bsp_status bsp_batch_default_options(bsp_batch_options *opt);
/* mats: host array of `count` descriptors (device pointers inside). */
bsp_status bsp_batch_create(int32_t count, const bsp_batch_mat *mats,
                            bsp_dtype dtype, int32_t nrhs,
                            const bsp_batch_options *opt, bsp_batch_plan *plan,
                            bsp_stream_t stream);
/* One launch for the whole batch (graph replay when use_graph). */
bsp_status bsp_batch_run(bsp_batch_plan plan, bsp_stream_t stream);
/* The same products as one plain kernel launch per matrix (comparison). */
bsp_status bsp_batch_run_separate(bsp_batch_plan plan, bsp_stream_t stream);
/* Replaces the x / y pointers of matrix m (no re-capture needed). */
bsp_status bsp_batch_set_vectors(bsp_batch_plan plan, int32_t m, const void *x,
                                 void *y, bsp_stream_t stream);
/* Per-matrix choice of the tuner: lanes per row (1..32) for CSR matrices,
 * 0 for matrices stored as SELL-32. */
bsp_status bsp_batch_lanes(bsp_batch_plan plan, int32_t *lanes /* count */);
/* Per-matrix storage: 0 = CSR, 1 = SELL-32 narrow form, 2 = SELL-32 wide form. */
bsp_status bsp_batch_formats(bsp_batch_plan plan, int32_t *formats /* count */);
bsp_status bsp_batch_stats(bsp_batch_plan plan, int64_t *items,
                           int64_t *long_segments, int64_t *total_nnz);
bsp_status bsp_batch_destroy(bsp_batch_plan plan);

/* ---------------------------------------------------------------------- */
/* Synthetic matrix generators (host, seeded, deterministic).  Two-phase:
 * call with NULL arrays to get the sizes, then with allocated arrays. */

/* 2-D 5-point Laplacian on an nx*ny grid, natural ordering, diag 4, off -1. */
bsp_status bsp_gen_laplace2d(int32_t nx, int32_t ny, int32_t *rows,
                             int32_t *nnz, int32_t *rowPtr, int32_t *colIdx,
                             double *values);
/* 3-D 7-point Poisson on n^3 (diag 6, off -1). */
bsp_status bsp_gen_poisson3d(int32_t n, int32_t *rows, int64_t *nnz,
                             int32_t *rowPtr, int32_t *colIdx, double *values);
/* 3-D 27-point stencil on n^3 nodes with `dof` unknowns per node: every
 * coupled node pair is a dense dof x dof block of N(0,1) values. */
bsp_status bsp_gen_stencil27(int32_t n, int32_t dof, uint64_t seed,
                             int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                             int32_t *colIdx, double *values);
/* Random block-sparse matrix: nbr block-rows of bs x bs blocks (bs 4, 8 or
 * 16), `per_row` distinct random block columns per block-row, each block
 * filled with probability U[fill_lo, fill_hi] per entry (at least one
 * entry). */
bsp_status bsp_gen_random_bsr(int32_t nbr, int32_t bs, int32_t per_row,
                              double fill_lo, double fill_hi, uint64_t seed,
                              int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                              int32_t *colIdx, double *values);
/* Power-law rows: row lengths ~ Zipf(alpha) on [1, max_len], distinct
 * uniform columns on [0, n), N(0,1) values. */
bsp_status bsp_gen_powerlaw(int32_t n, double alpha, int32_t max_len,
                            uint64_t seed, int32_t *rows, int64_t *nnz,
                            int32_t *rowPtr, int32_t *colIdx, double *values);
/* Power-law graph: out-degrees ~ Zipf(alpha) on [1, d_max], d_max chosen so
 * the mean degree is mean_deg; distinct uniform targets; values 1/degree. */
bsp_status bsp_gen_graph(int32_t n, double alpha, double mean_deg, uint64_t seed,
                         int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                         int32_t *colIdx, double *values);
/* Banded matrix: row i holds columns i-(width-1)/2 .. i+width/2 inside
 * [0, n), N(0,1) values. */
bsp_status bsp_gen_banded(int32_t n, int32_t width, uint64_t seed,
                          int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                          int32_t *colIdx, double *values);
/* Uniform random x in [-1, 1]. */
bsp_status bsp_gen_uniform(int64_t n, uint64_t seed, double *x);
/* SPD 7-point diffusion on an m^3 grid: face coefficients exp(contrast * u),
 * u ~ U[-1, 1] per face (Dirichlet boundary faces included on the diagonal);
 * contrast > 0 makes Jacobi preconditioning pay. */
bsp_status bsp_gen_diffusion3d(int32_t m, double contrast, uint64_t seed,
                               int32_t *rows, int64_t *nnz, int32_t *rowPtr,
                               int32_t *colIdx, double *values);
/* SPD block Laplacian L (x) S: L the 7-point diffusion with contrast 1, S a
 * seeded dof x dof SPD coupling with eigenvalues log-spaced in [1, cond];
 * node-major rows (dof consecutive rows per node), so block-Jacobi with
 * blocks of dof rows inverts S exactly. */
bsp_status bsp_gen_block_laplace3d(int32_t m, int32_t dof, double cond,
                                   uint64_t seed, int32_t *rows, int64_t *nnz,
                                   int32_t *rowPtr, int32_t *colIdx,
                                   double *values);

/* ---------------------------------------------------------------------- */
/* Matrix Market files.  Replaces the reference drivers' read_triplet_file +
 * triplet-to-CSR block (bench/spmvfp64.cpp:37-86, bench/spmvfp16.cpp:32-60,
 * bench/spmmfp16.cpp:32-60), which read through the third-party
 * fast_matrix_market header and then sort by (row, col).
 *
 * Accepted: "%%MatrixMarket matrix coordinate|array real|double|integer|pattern
 * general|symmetric|skew-symmetric|hermitian" (complex is BSP_ERR_UNSUPPORTED;
 * hermitian with a real field is symmetric).  Comment lines (%) and blank
 * lines may appear anywhere after the banner; CR-LF line ends are accepted.
 * Values are converted with correct rounding; pattern entries are 1.0.
 * Array files give every stored element (zeros included), column-major.
 *
 * Triplets are the file's entries in file order (1-based -> 0-based), then,
 * for a non-general file, one mirrored entry (j, i) per off-diagonal entry,
 * in file order, negated for skew-symmetric.  With BSP_MTX_DIAG_ZERO every
 * diagonal entry of a non-general file also gets an explicit 0.0 mirror,
 * which is fast_matrix_market's default element count (2 x entries);
 * BSP_MTX_DIAG_DUPLICATE repeats the diagonal value instead, and
 * BSP_MTX_NO_EXPAND keeps the stored entries only (its
 * generalize_symmetry = false).
 * CSR: rows ascending, columns ascending within a row, entries with the same
 * (row, col) kept in triplet order (duplicates are not summed). */
#define BSP_MTX_DIAG_ZERO 1      /* explicit 0.0 mirror per diagonal entry */
#define BSP_MTX_DIAG_DUPLICATE 2 /* a copy of each diagonal entry instead */
#define BSP_MTX_NO_EXPAND 4      /* stored entries only, no mirrors */

typedef enum { BSP_MTX_COORDINATE = 0, BSP_MTX_ARRAY = 1 } bsp_mtx_format;
typedef enum { BSP_MTX_REAL = 0, BSP_MTX_INTEGER = 1, BSP_MTX_PATTERN = 2 } bsp_mtx_field;
typedef enum {
  BSP_MTX_GENERAL = 0,
  BSP_MTX_SYMMETRIC = 1,
  BSP_MTX_SKEW_SYMMETRIC = 2,
  BSP_MTX_HERMITIAN = 3
} bsp_mtx_symmetry;

typedef struct {
  int64_t rows, cols;
  int64_t entries;  /* stored entries in the file */
  int64_t nnz;      /* triplets after the symmetry expansion */
  int32_t format, field, symmetry;
} bsp_mtx_info;

typedef struct bsp_mtx_s *bsp_mtx;

/* Maps and parses the whole file on `threads` host threads (0 = all).  The
 * handle keeps the triplets; rows, cols <= 2^31-1 and nnz <= 2^31-1. */
bsp_status bsp_mtx_read(const char *path, int32_t flags, int32_t threads,
                        bsp_mtx *out);
/* The same on file contents already in memory. */
bsp_status bsp_mtx_read_buffer(const char *data, size_t bytes, int32_t flags,
                               int32_t threads, bsp_mtx *out);
bsp_status bsp_mtx_get_info(bsp_mtx m, bsp_mtx_info *info);
/* The expanded triplets (nnz each), as read_matrix_market_triplet returns
 * them (any argument may be NULL to skip it). */
bsp_status bsp_mtx_triplets(bsp_mtx m, int32_t *rows, int32_t *cols,
                            double *values);
/* CSR on the host: rowPtr[rows+1], colIdx[nnz], values[nnz]. */
bsp_status bsp_mtx_csr_host(bsp_mtx m, int32_t *rowPtr, int32_t *colIdx,
                            double *values);
/* CSR in device memory (caller-allocated, same sizes): the triplets are
 * copied up and ordered on the device by two stable radix sorts. */
bsp_status bsp_mtx_csr(bsp_mtx m, int32_t *rowPtr, int32_t *colIdx,
                       double *values, bsp_stream_t stream);
bsp_status bsp_mtx_free(bsp_mtx m);
/* Writes host CSR as "coordinate real general" (values == NULL: "pattern"),
 * each value in its shortest round-trip decimal form. */
bsp_status bsp_mtx_write_csr_host(const char *path, int32_t rows, int32_t cols,
                                  int64_t nnz, const int32_t *rowPtr,
                                  const int32_t *colIdx, const double *values,
                                  int32_t threads);

#ifdef __cplusplus
}
#endif
#endif /* BSP_H */
