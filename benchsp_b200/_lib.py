"""ctypes binding of libbspmv.so (the C ABI declared in include/bsp.h).

Loading fails loudly: there is no CPU or PyTorch fallback behind these
entry points.  Build the library with ``python -m benchsp_b200.build``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libbspmv.so"

BSP_OK = 0
BSP_ERR_INVALID = 1
BSP_ERR_CUDA = 2
BSP_ERR_ALLOC = 3
BSP_ERR_NOT_CONVERGED = 4
BSP_ERR_UNSUPPORTED = 5
BSP_ERR_TIMEOUT = 6
STATUS_NAMES = {0: "BSP_OK", 1: "BSP_ERR_INVALID", 2: "BSP_ERR_CUDA", 3: "BSP_ERR_ALLOC",
                4: "BSP_ERR_NOT_CONVERGED", 5: "BSP_ERR_UNSUPPORTED", 6: "BSP_ERR_TIMEOUT"}

F64, F32, F16, BF16 = 0, 1, 2, 3

CSR_AUTO, CSR_VECTOR, CSR_MERGE, CSR_SCALAR, CSR_STREAM = 0, 1, 2, 3, 4
BSR_AUTO, BSR_FFMA, BSR_DMMA, BSR_ADAPTIVE = 0, 1, 2, 3


class BspError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class BspBsr(C.Structure):
    """Mirror of bsp_bsr (include/bsp.h), itself a mirror of the reference's
    bsrMAT (include/matrixFormat.hpp:59-83)."""
    _fields_ = [
        ("row", C.c_int32), ("col", C.c_int32), ("nnz", C.c_int32),
        ("blc_row", C.c_int32), ("blc_col", C.c_int32), ("blc_num", C.c_int32),
        ("stand", C.c_double), ("avg_nnz", C.c_double),
        ("blcPtr", C.c_void_p), ("blcIdx", C.c_void_p), ("blcVal", C.c_void_p), ("blcMap", C.c_void_p),
        ("warpnum", C.c_int32), ("rowPtrbyWarp", C.c_void_p), ("rowIdxbyWarp", C.c_void_p),
        ("bs", C.c_int32), ("true_nnz", C.c_int32), ("dense_blocks", C.c_int32),
    ]


class BspDbsr(C.Structure):
    """Mirror of bsp_dbsr (include/bsp.h), itself a mirror of the reference's
    dbsrMat (include/matrixFormat.hpp:86-106)."""
    _fields_ = [
        ("row", C.c_int32), ("col", C.c_int32), ("nnz", C.c_int32),
        ("blc_row", C.c_int32), ("blc_col", C.c_int32), ("blc_num", C.c_int32),
        ("stand", C.c_double), ("avg_nnz", C.c_double),
        ("blcPtr", C.c_void_p), ("colIdx", C.c_void_p), ("blcVal", C.c_void_p), ("blcMap", C.c_void_p),
        ("blocknnz", C.c_int32), ("warpnum", C.c_int32), ("rowPtrbyWarp", C.c_void_p),
        ("rowIdxbyWarp", C.c_void_p), ("recorderMap", C.c_void_p), ("prefix", C.c_void_p),
        ("balance_overflow", C.c_int32),
    ]


class BspBcsr(C.Structure):
    """Mirror of bsp_bcsr (include/bsp.h) / the reference's BCSRFormat
    (include/matrixFormat.hpp:16-30)."""
    _fields_ = [
        ("bcsrRowPtr", C.c_void_p), ("bcsrcolIdx", C.c_void_p), ("relativeBlockIndexMapping", C.c_void_p),
        ("values", C.c_void_p), ("row", C.c_int32), ("col", C.c_int32), ("blockNum", C.c_int64),
        ("TILE_M", C.c_int32), ("TILE_N", C.c_int32), ("TILE_K", C.c_int32), ("nnz", C.c_int32),
        ("colRegions", C.c_int32), ("rowRegions", C.c_int32), ("nonzeroBlocks", C.c_int32),
        ("elemCount", C.c_int32), ("block_row", C.c_int32), ("block_col", C.c_int32),
    ]


class BspDasp(C.Structure):
    """Mirror of bsp_dasp (include/bsp.h): the DASP packing of spmv_all
    (reference src/dasp.cu:814-1600)."""
    _fields_ = [
        ("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32), ("threshold", C.c_double),
        ("block_longest", C.c_int32), ("row_long", C.c_int32), ("row_block", C.c_int32), ("row_zero", C.c_int32),
        ("short_row_1", C.c_int32), ("short_row_2", C.c_int32), ("short_row_3", C.c_int32),
        ("short_row_4", C.c_int32), ("common_13", C.c_int32), ("short_row_34", C.c_int32),
        ("short_block13", C.c_int32), ("short_block34", C.c_int32), ("short_block22", C.c_int32),
        ("blocknum", C.c_int32), ("long_warps", C.c_int32), ("warp_number", C.c_int32),
        ("fill0_nnz_long", C.c_int32), ("fill0_nnz_short13", C.c_int32), ("fill0_nnz_short34", C.c_int32),
        ("fill0_nnz_short22", C.c_int32), ("fill0_nnz_short", C.c_int32), ("fill0_nnz_reg", C.c_int32),
        ("nnz_irreg", C.c_int32), ("offset_reg", C.c_int32), ("offset_short1", C.c_int32),
        ("offset_short13", C.c_int32), ("offset_short34", C.c_int32), ("offset_short22", C.c_int32),
        ("block_num_all", C.c_int32),
        ("long_val", C.c_void_p), ("long_cid", C.c_void_p), ("long_ptr_warp", C.c_void_p),
        ("long_row_of_warp", C.c_void_p), ("warp_val", C.c_void_p), ("long_done", C.c_void_p),
        ("reg_val", C.c_void_p), ("reg_cid", C.c_void_p), ("block_ptr", C.c_void_p),
        ("irreg_val", C.c_void_p), ("irreg_cid", C.c_void_p), ("irreg_rpt", C.c_void_p),
        ("short_val", C.c_void_p), ("short_cid", C.c_void_p), ("order_rid", C.c_void_p),
        ("sorted_rid", C.c_void_p), ("row_len_sorted", C.c_void_p),
        ("long_groups", C.c_int32), ("long_group_ptr", C.c_void_p), ("long_group_info", C.c_void_p),
    ]


_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_U64 = C.c_uint64
_D = C.c_double
_PI32 = C.POINTER(C.c_int32)
_PI64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes)
_PROTOS = {
    "bsp_last_error": (C.c_char_p, []),
    "bsp_version": (C.c_char_p, []),
    "bsp_memcpy_d2h": (C.c_int, [_P, _P, C.c_size_t]),
    "bsp_memcpy_h2d": (C.c_int, [_P, _P, C.c_size_t]),
    "bsp_device_sync": (C.c_int, []),
    "bsp_device_alloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    "bsp_device_free": (C.c_int, [_P]),
    "bsp_gather_probe": (C.c_int, [_P, C.c_size_t, _I32, _I64, _U64, _P, _P]),
    "bsp_csr_spmv": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, C.c_int, _P, _P, _D, _D, _I32, _I32, _P]),
    "bsp_csr_merge_workspace": (C.c_size_t, [_I32, _I32]),
    "bsp_csr_spmv_merge_f64": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _P, _P, _D, _D, _P, C.c_size_t, _P]),
    "bsp_csr_spmv_merge_f64_noalloc": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _P, _P, _D, _D, _P]),
    "bsp_csr2bsr": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _I32, C.POINTER(BspBsr), _P]),
    "bsp_bsr_free": (C.c_int, [C.POINTER(BspBsr)]),
    "bsp_bsr_spmv": (C.c_int, [C.POINTER(BspBsr), _P, _P, _D, _D, _I32, _P]),
    "bsp_bsr_spmv_variant": (C.c_int, [C.POINTER(BspBsr), _P, _P, _D, _D, _I32, _I32, _I32, _P]),
    "bsp_bsr_spmv_host": (C.c_int, [C.POINTER(BspBsr), _P, _P, _D, _D, _I32, _P]),
    "bsp_bsr_host_plan_create": (C.c_int, [C.POINTER(BspBsr), _I32, C.POINTER(C.c_void_p), _P]),
    "bsp_bsr_spmv_host_pipelined": (C.c_int, [C.c_void_p, _P, _P, _D, _D, _P]),
    "bsp_bsr_host_plan_destroy": (C.c_int, [C.c_void_p]),
    "bsp_bsr_host_plan_set_graph": (C.c_int, [C.c_void_p, _I32]),
    "bsp_bsr_host_plan_set_ctas": (C.c_int, [C.c_void_p, _I32]),
    "bsp_csr2bcsr": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _I32, _I32, _I32, C.POINTER(BspBcsr), _P]),
    "bsp_bcsr_free": (C.c_int, [C.POINTER(BspBcsr)]),
    "bsp_bcsr_spmv": (C.c_int, [C.POINTER(BspBcsr), _P, _P, _D, _D, _P]),
    "bsp_csr2dbsr": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _I32, C.POINTER(BspDbsr), _P]),
    "bsp_dbsr_free": (C.c_int, [C.POINTER(BspDbsr)]),
    "bsp_dbsr_spmv": (C.c_int, [C.POINTER(BspDbsr), _P, _P, _D, _D, _I32, _P]),
    "bsp_csr2dasp": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _D, _I32, C.POINTER(BspDasp), _P]),
    "bsp_dasp_free": (C.c_int, [C.POINTER(BspDasp)]),
    "bsp_dasp_spmv": (C.c_int, [C.POINTER(BspDasp), _P, _P, _D, _D, _I32, _P]),
    "bsp_blockinfo": (C.c_int, [_I32, _I32, _I32, _P, _P, _PI64, _PI64, _P]),
    "bsp_gen_laplace2d": (C.c_int, [_I32, _I32, _PI32, _PI32, _P, _P, _P]),
    "bsp_gen_poisson3d": (C.c_int, [_I32, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_stencil27": (C.c_int, [_I32, _I32, _U64, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_random_bsr": (C.c_int, [_I32, _I32, _I32, _D, _D, _U64, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_powerlaw": (C.c_int, [_I32, _D, _I32, _U64, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_uniform": (C.c_int, [_I64, _U64, _P]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m benchsp_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return list(_PROTOS)


def check(status: int) -> None:
    if status != BSP_OK:
        raise BspError(status, lib().bsp_last_error().decode(errors="replace"))


class BspCgOptions(C.Structure):
    """Mirror of bsp_cg_options (include/bsp.h)."""
    _fields_ = [("mode", C.c_int32), ("tol", C.c_double), ("max_iters", C.c_int32), ("check_every", C.c_int32),
                ("reliable_delta", C.c_double), ("use_graphs", C.c_int32), ("precond", C.c_int32),
                ("precond_block", C.c_int32), ("refine", C.c_int32)]


class BspSpmmChoice(C.Structure):
    _fields_ = [("engine", C.c_int32), ("smat_path", C.c_int32), ("reorder", C.c_int32), ("reserved", C.c_int32),
                ("tiles_given", C.c_int64), ("tiles_reordered", C.c_int64),
                ("est_seconds_smat_given", C.c_double), ("est_seconds_smat_reordered", C.c_double),
                ("est_seconds_csr", C.c_double), ("chunks_given", C.c_int64), ("chunks_reordered", C.c_int64),
                ("est_seconds_gtile_given", C.c_double), ("est_seconds_gtile_reordered", C.c_double)]


BSP_SPMM_ENGINE_CSR, BSP_SPMM_ENGINE_SMAT, BSP_SPMM_ENGINE_GTILE = 0, 1, 2


class BspCgResult(C.Structure):
    """Mirror of bsp_cg_result (include/bsp.h)."""
    _fields_ = [("iterations", C.c_int32), ("reliable_updates", C.c_int32), ("rel_residual", C.c_double),
                ("seconds", C.c_double), ("converged", C.c_int32), ("bytes_moved", C.c_int64),
                ("delta16", C.c_int32), ("outer_steps", C.c_int32)]


CG_FP64, CG_MIXED_F32, CG_MIXED_F16, CG_MIXED_BF16 = 0, 1, 2, 3

_PROTOS.update({
    "bsp_cg_default_options": (C.c_int, [C.POINTER(BspCgOptions)]),
    "bsp_cg_create": (C.c_int, [_I32, _I32, _P, _P, _P, C.POINTER(BspCgOptions), C.POINTER(C.c_void_p), _P]),
    "bsp_cg_solve": (C.c_int, [C.c_void_p, _P, _P, C.POINTER(BspCgResult), _P]),
    "bsp_cg_destroy": (C.c_int, [C.c_void_p]),
})


class BspSmat(C.Structure):
    """Mirror of bsp_smat (include/bsp.h)."""
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32), ("dtype", C.c_int32),
                ("tiles", BspBcsr), ("tile_val", C.c_void_p), ("err", C.c_void_p), ("fill", C.c_double)]


class BspBatchMat(C.Structure):
    """Mirror of bsp_batch_mat (include/bsp.h)."""
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32), ("rowPtr", C.c_void_p),
                ("colIdx", C.c_void_p), ("values", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p)]


class BspBatchOptions(C.Structure):
    """Mirror of bsp_batch_options (include/bsp.h)."""
    _fields_ = [("tune", C.c_int32), ("seg_nnz", C.c_int32), ("long_row_nnz", C.c_int32), ("item_nnz", C.c_int32),
                ("use_graph", C.c_int32), ("sell", C.c_int32), ("sell_wide", C.c_int32)]


_PROTOS.update({
    "bsp_batch_default_options": (C.c_int, [C.POINTER(BspBatchOptions)]),
    "bsp_batch_create": (C.c_int, [_I32, C.POINTER(BspBatchMat), C.c_int, _I32, C.POINTER(BspBatchOptions),
                                   C.POINTER(C.c_void_p), _P]),
    "bsp_batch_run": (C.c_int, [C.c_void_p, _P]),
    "bsp_batch_run_separate": (C.c_int, [C.c_void_p, _P]),
    "bsp_batch_set_vectors": (C.c_int, [C.c_void_p, _I32, _P, _P, _P]),
    "bsp_batch_lanes": (C.c_int, [C.c_void_p, _P]),
    "bsp_batch_formats": (C.c_int, [C.c_void_p, _P]),
    "bsp_batch_stats": (C.c_int, [C.c_void_p, _PI64, _PI64, _PI64]),
    "bsp_batch_destroy": (C.c_int, [C.c_void_p]),
    "bsp_gen_banded": (C.c_int, [_I32, _I32, _U64, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_diffusion3d": (C.c_int, [_I32, _D, _U64, _PI32, _PI64, _P, _P, _P]),
    "bsp_gen_block_laplace3d": (C.c_int, [_I32, _I32, _D, _U64, _PI32, _PI64, _P, _P, _P]),
})


class BspTuneResult(C.Structure):
    """Mirror of bsp_tune_result (include/bsp.h)."""
    _fields_ = [("format", C.c_int32), ("csr_algo", C.c_int32), ("lanes", C.c_int32), ("bs", C.c_int32),
                ("bsr_algo", C.c_int32), ("from_cache", C.c_int32), ("spmv_us", C.c_double), ("key", C.c_uint64),
                ("mean_len", C.c_double), ("cv_len", C.c_double), ("fill4", C.c_double), ("fill8", C.c_double),
                ("max_len", C.c_int32), ("long_rows", C.c_int32)]


FMT_CSR, FMT_BSR, FMT_DASP = 0, 1, 2

_PROTOS.update({
    "bsp_reorder_rcm": (C.c_int, [_I32, _I32, _P, _P, _P, _P]),
    "bsp_permute_csr": (C.c_int, [_I32, _I32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "bsp_reorder_rcm_host": (C.c_int, [_I32, _I32, _P, _P, _P]),
    "bsp_permute_csr_host": (C.c_int, [_I32, _I32, _P, _P, _P, _P, _P, _P, _P]),
    "bsp_reorder_similarity": (C.c_int, [_I32, _I32, _I32, _P, _P, _I32, _I32, _P, _P]),
    "bsp_reorder_similarity_host": (C.c_int, [_I32, _I32, _I32, _P, _P, _I32, _I32, _P]),
    "bsp_permute_rows_csr": (C.c_int, [_I32, _I32, _P, _P, _P, _P, _P, _P, _P, _P]),
    "bsp_permute_rows_csr_host": (C.c_int, [_I32, _I32, _P, _P, _P, _P, _P, _P, _P]),
    "bsp_spmm_choose_host": (C.c_int, [_I32, _I32, _I32, _P, _P, _I32, _P, C.POINTER(BspSpmmChoice)]),
})

_PROTOS.update({
    "bsp_tune_spmv": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _I32, C.POINTER(BspTuneResult), _P]),
    "bsp_matrix_key": (C.c_int, [_I32, _I32, _I32, _P, _P, C.POINTER(C.c_uint64), _P]),
    "bsp_tune_cache_clear": (None, []),
    "bsp_spmv_plan_create": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, _I32, C.POINTER(C.c_void_p), _P]),
    "bsp_spmv_plan_choice": (C.c_int, [C.c_void_p, C.POINTER(BspTuneResult)]),
    "bsp_spmv_plan_run": (C.c_int, [C.c_void_p, _P, _P, _D, _D, _P]),
    "bsp_spmv_plan_destroy": (C.c_int, [C.c_void_p]),
})


class BspSpmmPlan(C.Structure):
    """Mirror of bsp_spmm_plan (include/bsp.h)."""
    _fields_ = [("rows", C.c_int32), ("chunk", C.c_int32), ("nchunks", C.c_int64), ("nparts", C.c_int64),
                ("nsplit", C.c_int32), ("chunk_ptr", C.c_void_p), ("part_ptr", C.c_void_p),
                ("chunk_row", C.c_void_p), ("split_rows", C.c_void_p), ("nshort", C.c_int32),
                ("short_rows", C.c_void_p), ("long_chunk", C.c_void_p), ("long_se", C.c_void_p),
                ("short_se", C.c_void_p), ("slab_l2_hints", C.c_int32), ("ngroups", C.c_int32),
                ("group_ptr", C.c_void_p), ("group_split", C.c_void_p)]


_PROTOS.update({
    "bsp_spmm_plan_create": (C.c_int, [_I32, _I32, _P, _I32, C.POINTER(BspSpmmPlan), _P]),
    "bsp_spmm_plan_free": (C.c_int, [C.POINTER(BspSpmmPlan)]),
    "bsp_spmm_plan_workspace": (C.c_size_t, [C.POINTER(BspSpmmPlan), _I32]),
    "bsp_spmm_csr_planned": (C.c_int, [C.POINTER(BspSpmmPlan), _I32, _I32, _P, _P, _P, C.c_int, _P, _I32, _I64, _P,
                                       _I64, C.c_float, C.c_float, _P, C.c_size_t, _P]),
    "bsp_spmm_csr_planned_variant": (C.c_int, [C.POINTER(BspSpmmPlan), _I32, _I32, _P, _P, _P, C.c_int, _P, _I32,
                                               _I64, _P, _I64, C.c_float, C.c_float, _P, C.c_size_t, _I32, _I32,
                                               _P]),
    "bsp_spmm_csr": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, C.c_int, _P, _I32, _I64, _P, _I64, C.c_float,
                               C.c_float, _P]),
    "bsp_smat_create": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, C.c_int, C.POINTER(BspSmat), _P]),
    "bsp_smat_free": (C.c_int, [C.POINTER(BspSmat)]),
    "bsp_smat_spmm": (C.c_int, [C.POINTER(BspSmat), _P, _I32, _I64, _P, _I64, C.c_float, C.c_float, _P]),
    "bsp_smat_check": (C.c_int, [C.POINTER(BspSmat), _P]),
    "bsp_smat_spmm_path": (C.c_int, [C.POINTER(BspSmat), _P, _I32, _I64, _P, _I64, C.c_float, C.c_float, _I32,
                                     _P]),
    "bsp_gen_graph": (C.c_int, [_I32, _D, _D, _U64, _PI32, _PI64, _P, _P, _P]),
})


class BspMtxInfo(C.Structure):
    """Mirror of bsp_mtx_info (include/bsp.h)."""
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("entries", C.c_int64), ("nnz", C.c_int64),
                ("format", C.c_int32), ("field", C.c_int32), ("symmetry", C.c_int32)]


MTX_DIAG_ZERO, MTX_DIAG_DUPLICATE, MTX_NO_EXPAND = 1, 2, 4

_PROTOS.update({
    "bsp_mtx_read": (C.c_int, [C.c_char_p, _I32, _I32, C.POINTER(C.c_void_p)]),
    "bsp_mtx_read_buffer": (C.c_int, [C.c_char_p, C.c_size_t, _I32, _I32, C.POINTER(C.c_void_p)]),
    "bsp_mtx_get_info": (C.c_int, [C.c_void_p, C.POINTER(BspMtxInfo)]),
    "bsp_mtx_triplets": (C.c_int, [C.c_void_p, _P, _P, _P]),
    "bsp_mtx_csr_host": (C.c_int, [C.c_void_p, _P, _P, _P]),
    "bsp_mtx_csr": (C.c_int, [C.c_void_p, _P, _P, _P, _P]),
    "bsp_mtx_free": (C.c_int, [C.c_void_p]),
    "bsp_mtx_write_csr_host": (C.c_int, [C.c_char_p, _I32, _I32, _I64, _P, _P, _P, _I32]),
})

_PROTOS.update({
    "bsp_cg_solve_multi": (C.c_int, [C.c_void_p, _I32, _P, _I64, _P, _I64, _P, C.POINTER(BspCgResult), _P]),
})


class BspBsrScaled(C.Structure):
    """Mirror of bsp_bsr_scaled (include/bsp.h): FP16/BF16 BSR with one
    power-of-two scale per block."""
    _fields_ = [
        ("row", C.c_int32), ("col", C.c_int32), ("bs", C.c_int32),
        ("blc_row", C.c_int32), ("blc_col", C.c_int32), ("blc_num", C.c_int32),
        ("dtype", C.c_int32), ("blcPtr", C.c_void_p), ("blcKey", C.c_void_p), ("blcVal", C.c_void_p),
    ]


_PROTOS.update({
    "bsp_bsr_scaled_create": (C.c_int, [C.POINTER(BspBsr), _I32, C.POINTER(BspBsrScaled), _P]),
    "bsp_bsr_scaled_free": (C.c_int, [C.POINTER(BspBsrScaled)]),
    "bsp_bsr_scaled_spmv": (C.c_int, [C.POINTER(BspBsrScaled), _P, _I32, _P, _I32, _D, _D, _P]),
    "bsp_bsr_scaled_spmv_variant": (C.c_int, [C.POINTER(BspBsrScaled), _P, _I32, _P, _I32, _D, _D, _I32, _I32,
                                              _P]),
})


class BspGtile(C.Structure):
    """Mirror of bsp_gtile (include/bsp.h): gathered-tile SpMM matrix."""
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32), ("dtype", C.c_int32),
                ("nchunks", C.c_int64), ("ngroups", C.c_int32), ("npieces", C.c_int32), ("nsplit", C.c_int32),
                ("nslots", C.c_int32), ("piece_ptr", C.c_void_p), ("piece_group", C.c_void_p),
                ("piece_slot", C.c_void_p), ("group_piece", C.c_void_p), ("split_groups", C.c_void_p),
                ("chunk_cols", C.c_void_p), ("chunk_tiles", C.c_void_p), ("err", C.c_void_p)]


_PROTOS.update({
    "bsp_gtile_create_host": (C.c_int, [_I32, _I32, _I32, _P, _P, _P, C.c_int, C.POINTER(BspGtile)]),
    "bsp_gtile_workspace": (C.c_size_t, [C.POINTER(BspGtile), _I32]),
    "bsp_gtile_spmm": (C.c_int, [C.POINTER(BspGtile), _P, _I32, _I64, _P, _I64, C.c_float, C.c_float, _P,
                                 C.c_size_t, _P]),
    "bsp_gtile_check": (C.c_int, [C.POINTER(BspGtile), _P]),
    "bsp_gtile_free": (C.c_int, [C.POINTER(BspGtile)]),
})
