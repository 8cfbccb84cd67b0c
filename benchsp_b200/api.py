"""Python host API over the C ABI (include/bsp.h).

Device memory and streams come from PyTorch (plumbing only); every
operation runs in libbspmv's CUDA kernels.  Names and argument meaning
follow the reference's operator surface (jiajun-c/benchsp include/*.h):
CSR SpMV (csrspmv.h / spmv.h), AmgT BSR (amgT.h, bsrMAT), and the
synthetic inputs stand in for its .mtx matrices.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import BspBsr, check, lib

_ALGO_CSR = {"auto": _lib.CSR_AUTO, "vector": _lib.CSR_VECTOR, "merge": _lib.CSR_MERGE,
             "scalar": _lib.CSR_SCALAR, "stream": _lib.CSR_STREAM}
_ALGO_BSR = {"auto": _lib.BSR_AUTO, "ffma": _lib.BSR_FFMA, "dmma": _lib.BSR_DMMA,
             "adaptive": _lib.BSR_ADAPTIVE}


def _torch():
    import torch
    return torch


def _stream(stream=None) -> C.c_void_p:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dptr(t, name: str) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return C.c_void_p(t.data_ptr())


def _dtype_code(t) -> int:
    torch = _torch()
    m = {torch.float64: _lib.F64, torch.float32: _lib.F32, torch.float16: _lib.F16,
         torch.bfloat16: _lib.BF16}
    if t.dtype not in m:
        raise ValueError(f"unsupported dtype {t.dtype}")
    return m[t.dtype]


# ---------------------------------------------------------------------------
# CSR SpMV (replaces spmv_fp64_warpper / spmv_fp64_balance_warpper,
# reference src/csrspmv.cu:104,136, and MySpmvWithPrefp64/fp16, src/spmv.cu)

def csr_spmv(rowptr, colidx, values, x, y=None, *, rows: int | None = None, cols: int | None = None,
             alpha: float = 1.0, beta: float = 0.0, algo: str = "auto", lanes: int = 0, stream=None):
    """y = alpha*A*x + beta*y for int32 CSR on the device; returns y."""
    torch = _torch()
    rows = rowptr.numel() - 1 if rows is None else rows
    cols = x.numel() if cols is None else cols
    nnz = colidx.numel()
    if y is None:
        y = torch.empty(rows, dtype=values.dtype, device=values.device)
        beta = 0.0
    dt = _dtype_code(values)
    if x.dtype != values.dtype or y.dtype != values.dtype:
        raise ValueError("values, x and y must share a dtype")
    check(lib().bsp_csr_spmv(rows, cols, nnz, _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                             _dptr(values, "values"), dt, _dptr(x, "x"), _dptr(y, "y"), float(alpha),
                             float(beta), _ALGO_CSR[algo], int(lanes), _stream(stream)))
    return y


def csr_merge_workspace_bytes(rows: int, nnz: int) -> int:
    return int(lib().bsp_csr_merge_workspace(rows, nnz))


def csr_spmv_merge(rowptr, colidx, values, x, y=None, *, workspace=None, alpha: float = 1.0,
                   beta: float = 0.0, stream=None):
    """FP64 merge-path SpMV with an explicit (caller-owned) workspace."""
    torch = _torch()
    rows = rowptr.numel() - 1
    nnz = colidx.numel()
    if y is None:
        y = torch.empty(rows, dtype=torch.float64, device=values.device)
        beta = 0.0
    need = csr_merge_workspace_bytes(rows, nnz)
    if workspace is None:
        workspace = torch.empty(need, dtype=torch.uint8, device=values.device)
    check(lib().bsp_csr_spmv_merge_f64(rows, x.numel(), nnz, _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                       _dptr(values, "values"), _dptr(x, "x"), _dptr(y, "y"), float(alpha),
                                       float(beta), _dptr(workspace, "workspace"), workspace.numel(),
                                       _stream(stream)))
    return y


# ---------------------------------------------------------------------------
# AmgT BSR (bsrMAT, reference include/matrixFormat.hpp:59-83; CSR2BSR_GPU,
# src/amgT.cu:1114; amgT_spmv_fp64, src/amgT.cu:1355)

def _d2h(ptr: int, count: int, dtype) -> np.ndarray:
    out = np.empty(count, dtype=dtype)
    if count:
        check(lib().bsp_memcpy_d2h(out.ctypes.data_as(C.c_void_p), C.c_void_p(ptr), out.nbytes))
    return out


def _host_vec(a, n: int, name: str) -> None:
    """The host-buffer calls copy n doubles to or from `a`: it must be a
    C-contiguous float64 numpy array of at least n entries."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError(f"{name} must be a C-contiguous float64 numpy array")
    if a.size < n:
        raise ValueError(f"{name} has {a.size} entries, the matrix needs {n}")


class BsrMatrix:
    """Device BSR matrix built by the library (bs = 4 reproduces bsrMAT)."""

    def __init__(self, desc: BspBsr):
        self._d = desc
        self._live = True

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(BspBsr._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    @property
    def desc(self) -> BspBsr:
        return self._d

    def arrays(self) -> dict[str, np.ndarray]:
        """Copies every array to host numpy arrays."""
        d = self._d
        maptype = np.uint16 if d.bs == 4 else np.uint64
        return {
            "blcPtr": _d2h(d.blcPtr, d.blc_row + 1, np.int32),
            "blcIdx": _d2h(d.blcIdx, d.blc_num, np.int32),
            "blcVal": _d2h(d.blcVal, d.blc_num * d.bs * d.bs, np.float64),
            "blcMap": _d2h(d.blcMap, d.blc_num, maptype),
            "rowPtrbyWarp": _d2h(d.rowPtrbyWarp, d.blc_row + 1, np.int32),
            "rowIdxbyWarp": _d2h(d.rowIdxbyWarp, d.warpnum, np.int32),
        }

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, algo: str = "auto", stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self._d.row, dtype=torch.float64, device=x.device)
            beta = 0.0
        check(lib().bsp_bsr_spmv(C.byref(self._d), _dptr(x, "x"), _dptr(y, "y"), float(alpha), float(beta),
                                 _ALGO_BSR[algo], _stream(stream)))
        return y

    def spmv_variant(self, x, y, *, lanes: int, unroll: int, l2_prefetch: int = 0, alpha: float = 1.0,
                     beta: float = 0.0, stream=None):
        """FFMA SpMV with an explicit kernel shape (autotuner candidates)."""
        check(lib().bsp_bsr_spmv_variant(C.byref(self._d), _dptr(x, "x"), _dptr(y, "y"), float(alpha),
                                         float(beta), lanes, unroll, l2_prefetch, _stream(stream)))
        return y

    def spmv_host(self, x_host: np.ndarray, y_host: np.ndarray, *, alpha: float = 1.0, beta: float = 0.0,
                  algo: str = "auto", stream=None) -> np.ndarray:
        """Host-buffer SpMV (H2D x, SpMV, D2H y, wait); x_host/y_host are
        float64 numpy arrays, ideally in pinned memory."""
        _host_vec(x_host, self._d.col, "x_host")
        _host_vec(y_host, self._d.row, "y_host")
        check(lib().bsp_bsr_spmv_host(C.byref(self._d), C.c_void_p(x_host.ctypes.data),
                                      C.c_void_p(y_host.ctypes.data), float(alpha), float(beta), _ALGO_BSR[algo],
                                      _stream(stream)))
        return y_host

    def scaled(self, dtype: str = "f16", stream=None) -> "BsrScaledMatrix":
        """FP16/BF16 copy with one power-of-two scale per block."""
        return BsrScaledMatrix(self, dtype, stream)

    def host_plan(self, chunks: int = 8, stream=None, use_graph: bool = True) -> "BsrHostPlan":
        """Overlapped host-buffer SpMV plan (see BsrHostPlan)."""
        return BsrHostPlan(self, chunks, stream, use_graph)

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_bsr_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BsrHostPlan:
    """Host-buffer BSR SpMV with the x upload, the SpMV and the y download
    overlapped in block-row chunks (keeps the matrix alive)."""

    def __init__(self, M: "BsrMatrix", chunks: int = 8, stream=None, use_graph: bool = True):
        self._m = M
        self._h = C.c_void_p()
        check(lib().bsp_bsr_host_plan_create(C.byref(M._d), chunks, C.byref(self._h), _stream(stream)))
        if not use_graph:
            check(lib().bsp_bsr_host_plan_set_graph(self._h, 0))

    def set_ctas(self, max_ctas: int) -> None:
        """Caps each range's SpMV grid (0 = the kernel's own; the plan
        starts at one wave, 8 CTAs per SM)."""
        check(lib().bsp_bsr_host_plan_set_ctas(self._h, int(max_ctas)))

    def spmv(self, x_host: np.ndarray, y_host: np.ndarray, *, alpha: float = 1.0, beta: float = 0.0,
             stream=None) -> np.ndarray:
        _host_vec(x_host, self._m._d.col, "x_host")
        _host_vec(y_host, self._m._d.row, "y_host")
        check(lib().bsp_bsr_spmv_host_pipelined(self._h, x_host.ctypes.data_as(C.c_void_p),
                                                y_host.ctypes.data_as(C.c_void_p), float(alpha), float(beta),
                                                _stream(stream)))
        return y_host

    def close(self) -> None:
        if self._h:
            check(lib().bsp_bsr_host_plan_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BsrScaledMatrix:
    """FP16/BF16 BSR with one power-of-two scale per block (bsp_bsr_scaled),
    built from a BsrMatrix; the source may be freed afterwards."""

    _DT = {"f16": _lib.F16, "bf16": _lib.BF16}

    def __init__(self, src: "BsrMatrix", dtype: str = "f16", stream=None):
        self._d = _lib.BspBsrScaled()
        check(lib().bsp_bsr_scaled_create(C.byref(src._d), self._DT[dtype], C.byref(self._d), _stream(stream)))
        self._live = True

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(_lib.BspBsrScaled._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    def stored_bytes(self) -> int:
        """Bytes of the matrix arrays (values, keys, block-row pointers)."""
        d = self._d
        return d.blc_num * d.bs * d.bs * 2 + d.blc_num * 4 + (d.blc_row + 1) * 4

    def arrays(self) -> dict[str, np.ndarray]:
        d = self._d
        return {"blcPtr": _d2h(d.blcPtr, d.blc_row + 1, np.int32),
                "blcKey": _d2h(d.blcKey, d.blc_num, np.uint32),
                "blcVal": _d2h(d.blcVal, d.blc_num * d.bs * d.bs, np.uint16)}

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, lanes: int = 0, unroll: int = 1,
             stream=None):
        """y = alpha*A*x + beta*y; x and y float64 or float32 device tensors
        (y defaults to x's dtype); FP32 products and sums."""
        torch = _torch()
        if y is None:
            y = torch.empty(self._d.row, dtype=x.dtype, device=x.device)
            beta = 0.0
        codes = {torch.float64: _lib.F64, torch.float32: _lib.F32}
        if x.dtype not in codes or y.dtype not in codes:
            raise ValueError("x and y must be float64 or float32")
        if x.numel() < self._d.col or y.numel() < self._d.row:
            raise ValueError("x or y is shorter than the matrix")
        if lanes:
            check(lib().bsp_bsr_scaled_spmv_variant(C.byref(self._d), _dptr(x, "x"), codes[x.dtype], _dptr(y, "y"),
                                                    codes[y.dtype], float(alpha), float(beta), lanes, unroll,
                                                    _stream(stream)))
        else:
            check(lib().bsp_bsr_scaled_spmv(C.byref(self._d), _dptr(x, "x"), codes[x.dtype], _dptr(y, "y"),
                                            codes[y.dtype], float(alpha), float(beta), _stream(stream)))
        return y

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_bsr_scaled_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr2bsr(rowptr, colidx, values, *, rows: int, cols: int, bs: int = 4, stream=None) -> BsrMatrix:
    d = BspBsr()
    check(lib().bsp_csr2bsr(rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                            _dptr(values, "values"), bs, C.byref(d), _stream(stream)))
    return BsrMatrix(d)


# ---------------------------------------------------------------------------
# Fixed-tile BCSR (BCSRFormat, reference include/matrixFormat.hpp:16-30;
# csrToBcsr, utils/utils.hpp:10; bcsr_spmv_fp64, src/bcsr.cu:224)

class BcsrMatrix:
    def __init__(self, desc: _lib.BspBcsr):
        self._d = desc
        self._live = True

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(_lib.BspBcsr._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    def arrays(self) -> dict[str, np.ndarray]:
        d = self._d
        out = {"bcsrRowPtr": _d2h(d.bcsrRowPtr, d.rowRegions + 1, np.int32),
               "bcsrColIdx": _d2h(d.bcsrcolIdx, d.nonzeroBlocks, np.int32),
               "bcsrVal": _d2h(d.values, d.elemCount, np.float64)}
        if d.relativeBlockIndexMapping:
            out["mapping"] = _d2h(d.relativeBlockIndexMapping, d.blockNum, np.int32)
        return out

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self._d.row, dtype=torch.float64, device=x.device)
            beta = 0.0
        check(lib().bsp_bcsr_spmv(C.byref(self._d), _dptr(x, "x"), _dptr(y, "y"), float(alpha), float(beta),
                                  _stream(stream)))
        return y

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_bcsr_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr2bcsr(rowptr, colidx, values, *, rows: int, cols: int, tile_m: int, tile_k: int, mapping: bool = False,
             stream=None) -> BcsrMatrix:
    d = _lib.BspBcsr()
    check(lib().bsp_csr2bcsr(rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                             _dptr(values, "values"), tile_m, tile_k, int(mapping), C.byref(d), _stream(stream)))
    return BcsrMatrix(d)


# ---------------------------------------------------------------------------
# DBSR (dbsrMat, reference include/matrixFormat.hpp:86-106; csrTodbsr /
# csrTodbsrWithRecorder / balanceDbsr, include/dbsr.h; amgT_spmv_fp64_dbsr*,
# src/amgT.cu:1202-1353)

class DbsrMatrix:
    """Device DBSR matrix (4x4 blocks of consecutive nonzeros per row quad)."""

    def __init__(self, desc: _lib.BspDbsr):
        self._d = desc
        self._live = True

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(_lib.BspDbsr._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    def arrays(self) -> dict[str, np.ndarray]:
        d = self._d
        out = {
            "blcPtr": _d2h(d.blcPtr, d.blc_row + 1, np.int32),
            "colIdx": _d2h(d.colIdx, d.blocknnz, np.int32),
            "blcVal": _d2h(d.blcVal, d.blocknnz, np.float64),
            "blcMap": _d2h(d.blcMap, d.blc_num, np.uint16),
            "prefix": _d2h(d.prefix, d.warpnum + 1, np.int32),
        }
        if d.recorderMap:
            out["recorderMap"] = _d2h(d.recorderMap, d.row, np.int32)
        return out

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, permuted: bool = False, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self._d.row, dtype=torch.float64, device=x.device)
            beta = 0.0
        check(lib().bsp_dbsr_spmv(C.byref(self._d), _dptr(x, "x"), _dptr(y, "y"), float(alpha), float(beta),
                                  int(permuted), _stream(stream)))
        return y

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_dbsr_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr2dbsr(rowptr, colidx, values, *, rows: int, cols: int, recorder: bool = True, stream=None) -> DbsrMatrix:
    d = _lib.BspDbsr()
    check(lib().bsp_csr2dbsr(rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                             _dptr(values, "values"), int(recorder), C.byref(d), _stream(stream)))
    return DbsrMatrix(d)


# ---------------------------------------------------------------------------
# DASP (spmv_all, reference src/dasp.cu:814; include/dasp.h)

class DaspMatrix:
    """Device DASP packing (long / row-block / short row classes)."""

    INT_FIELDS = ("row_long", "row_block", "row_zero", "short_row_1", "short_row_2", "short_row_3", "short_row_4",
                  "common_13", "short_row_34", "blocknum", "warp_number", "fill0_nnz_long", "fill0_nnz_short13",
                  "fill0_nnz_short34", "fill0_nnz_short22", "fill0_nnz_short", "fill0_nnz_reg", "nnz_irreg",
                  "offset_reg", "offset_short1", "offset_short13", "offset_short34", "offset_short22",
                  "block_num_all")

    def __init__(self, desc: _lib.BspDasp):
        self._d = desc
        self._live = True

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(_lib.BspDasp._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    def arrays(self) -> dict[str, np.ndarray]:
        d = self._d
        return {
            "long_val": _d2h(d.long_val, d.fill0_nnz_long, np.float64),
            "long_cid": _d2h(d.long_cid, d.fill0_nnz_long, np.int32),
            "long_ptr_warp": _d2h(d.long_ptr_warp, d.row_long + 1, np.int32),
            "reg_val": _d2h(d.reg_val, d.fill0_nnz_reg, np.float64),
            "reg_cid": _d2h(d.reg_cid, d.fill0_nnz_reg, np.int32),
            "block_ptr": _d2h(d.block_ptr, d.blocknum + 1, np.int32),
            "irreg_val": _d2h(d.irreg_val, d.nnz_irreg, np.float64),
            "irreg_cid": _d2h(d.irreg_cid, d.nnz_irreg, np.int32),
            "irreg_rpt": _d2h(d.irreg_rpt, d.row_block + 1, np.int32),
            "short_val": _d2h(d.short_val, d.fill0_nnz_short, np.float64),
            "short_cid": _d2h(d.short_cid, d.fill0_nnz_short, np.int32),
            "order_rid": _d2h(d.order_rid, d.rows, np.int32),
        }

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, permuted: bool = False, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self._d.rows, dtype=torch.float64, device=x.device)
            beta = 0.0
        check(lib().bsp_dasp_spmv(C.byref(self._d), _dptr(x, "x"), _dptr(y, "y"), float(alpha), float(beta),
                                  int(permuted), _stream(stream)))
        return y

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_dasp_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr2dasp(rowptr, colidx, values, *, rows: int, cols: int, threshold: float = 0.75, block_longest: int = 256,
             stream=None) -> DaspMatrix:
    d = _lib.BspDasp()
    check(lib().bsp_csr2dasp(rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                             _dptr(values, "values"), float(threshold), int(block_longest), C.byref(d),
                             _stream(stream)))
    return DaspMatrix(d)


# ---------------------------------------------------------------------------
# Block statistics (reference bench/blockinfo.cpp:96-119)

def blockinfo(rowptr, colidx, *, rows: int, cols: int, stream=None) -> dict:
    """Distinct 4x4 blocks without / with the row-packed (recorder) layout."""
    b = C.c_int64()
    br = C.c_int64()
    nnz = colidx.numel()
    check(lib().bsp_blockinfo(rows, cols, nnz, _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"), C.byref(b),
                              C.byref(br), _stream(stream)))
    return {"blocks": b.value, "blocks_recorder": br.value,
            "avg_nnz": nnz / b.value if b.value else 0.0,
            "avg_nnz_recorder": nnz / br.value if br.value else 0.0}


# ---------------------------------------------------------------------------
# Seeded synthetic inputs (host numpy arrays)

@dataclass
class HostCSR:
    rows: int
    cols: int
    rowptr: np.ndarray
    colidx: np.ndarray
    values: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.colidx.size)

    def to_device(self, device="cuda"):
        torch = _torch()
        return (torch.from_numpy(self.rowptr).to(device), torch.from_numpy(self.colidx).to(device),
                torch.from_numpy(self.values).to(device))


def _two_phase(fn, *head) -> HostCSR:
    rows = C.c_int32()
    nnz = C.c_int64()
    check(fn(*head, C.byref(rows), C.byref(nnz), None, None, None))
    rp = np.empty(rows.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    va = np.empty(nnz.value, np.float64)
    check(fn(*head, C.byref(rows), C.byref(nnz), rp.ctypes.data_as(C.c_void_p), ci.ctypes.data_as(C.c_void_p),
             va.ctypes.data_as(C.c_void_p)))
    return HostCSR(rows.value, rows.value, rp, ci, va)


def gen_laplace2d(nx: int, ny: int) -> HostCSR:
    rows = C.c_int32()
    nnz = C.c_int32()
    L = lib()
    check(L.bsp_gen_laplace2d(nx, ny, C.byref(rows), C.byref(nnz), None, None, None))
    rp = np.empty(rows.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    va = np.empty(nnz.value, np.float64)
    check(L.bsp_gen_laplace2d(nx, ny, C.byref(rows), C.byref(nnz), rp.ctypes.data_as(C.c_void_p),
                              ci.ctypes.data_as(C.c_void_p), va.ctypes.data_as(C.c_void_p)))
    return HostCSR(rows.value, rows.value, rp, ci, va)


def gen_poisson3d(n: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_poisson3d, n)


def gen_diffusion3d(n: int, contrast: float, seed: int) -> HostCSR:
    """SPD 7-point diffusion, face coefficients exp(contrast * U[-1, 1])."""
    return _two_phase(lib().bsp_gen_diffusion3d, n, float(contrast), seed)


def gen_block_laplace3d(n: int, dof: int, cond: float, seed: int) -> HostCSR:
    """SPD L (x) S with a dof x dof coupling S of condition number `cond`."""
    return _two_phase(lib().bsp_gen_block_laplace3d, n, dof, float(cond), seed)


def gen_stencil27(n: int, dof: int, seed: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_stencil27, n, dof, seed)


def gen_random_bsr(nbr: int, bs: int, per_row: int, fill_lo: float, fill_hi: float, seed: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_random_bsr, nbr, bs, per_row, fill_lo, fill_hi, seed)


def gen_powerlaw(n: int, alpha: float, max_len: int, seed: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_powerlaw, n, alpha, max_len, seed)


def gen_uniform(n: int, seed: int) -> np.ndarray:
    x = np.empty(n, np.float64)
    check(lib().bsp_gen_uniform(n, seed, x.ctypes.data_as(C.c_void_p)))
    return x


# ---------------------------------------------------------------------------
# Conjugate gradients: FP64, or mixed precision with FP64 refinement

_CG_MODES = {"fp64": _lib.CG_FP64, "f32": _lib.CG_MIXED_F32, "f16": _lib.CG_MIXED_F16, "bf16": _lib.CG_MIXED_BF16}


_CG_PRECONDS = {"none": 0, "jacobi": 1, "block_jacobi": 2}


class CgSolver:
    """Solver plan for an SPD CSR matrix on the device (arrays must stay alive)."""

    def __init__(self, rowptr, colidx, values, *, mode: str = "f16", tol: float = 1e-10, max_iters: int = 20000,
                 check_every: int = 16, reliable_delta: float = 0.1, use_graphs: bool = True,
                 precond: str = "none", block: int = 4, refine: str = "auto", stream=None):
        """precond: "none", "jacobi" or "block_jacobi" (diagonal blocks of `block` rows, 4 or 8);
        refine (mixed modes): "auto", "reliable" or "flexible"."""
        o = _lib.BspCgOptions()
        check(lib().bsp_cg_default_options(C.byref(o)))
        o.mode, o.tol, o.max_iters, o.check_every = _CG_MODES[mode], tol, max_iters, check_every
        o.reliable_delta, o.use_graphs = reliable_delta, int(use_graphs)
        o.precond, o.precond_block = _CG_PRECONDS[precond], int(block)
        o.refine = {"auto": 0, "reliable": 1, "flexible": 2}[refine]
        self._keep = (rowptr, colidx, values)
        self.n = rowptr.numel() - 1
        self._plan = C.c_void_p()
        check(lib().bsp_cg_create(self.n, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                  _dptr(values, "values"), C.byref(o), C.byref(self._plan), _stream(stream)))

    def solve(self, b, x=None, *, stream=None, raise_on_stall: bool = True) -> tuple:
        torch = _torch()
        if x is None:
            x = torch.zeros(self.n, dtype=torch.float64, device=b.device)
        r = _lib.BspCgResult()
        st = lib().bsp_cg_solve(self._plan, _dptr(b, "b"), _dptr(x, "x"), C.byref(r), _stream(stream))
        if st != _lib.BSP_ERR_NOT_CONVERGED or raise_on_stall:
            check(st)
        return x, {k: getattr(r, k) for k, _ in _lib.BspCgResult._fields_}

    def solve_multi(self, B, X=None, *, stream=None, raise_on_stall: bool = True) -> tuple:
        """A X = B for the k columns of B (n x k, FP64, row-major); FP64
        plans with no or Jacobi preconditioning.  Returns (X, per-column
        relative residuals, aggregate result)."""
        torch = _torch()
        k = B.shape[1]
        if X is None:
            X = torch.zeros(self.n, k, dtype=torch.float64, device=B.device)
        for t, nm in ((B, "B"), (X, "X")):
            if not t.is_cuda or t.dtype != torch.float64 or t.dim() != 2 or t.shape[0] != self.n or \
                    (t.shape[1] > 1 and t.stride(1) != 1):
                raise ValueError(f"{nm} must be a row-major n x k FP64 CUDA tensor (column stride 1)")
        if X.shape[1] != k:
            raise ValueError("X must have as many columns as B")
        rel = np.zeros(k)
        r = _lib.BspCgResult()
        st = lib().bsp_cg_solve_multi(self._plan, k, C.c_void_p(B.data_ptr()), max(B.stride(0), k),
                                      C.c_void_p(X.data_ptr()), max(X.stride(0), k),
                                      rel.ctypes.data_as(C.c_void_p), C.byref(r), _stream(stream))
        if st != _lib.BSP_ERR_NOT_CONVERGED or raise_on_stall:
            check(st)
        return X, rel, {k2: getattr(r, k2) for k2, _ in _lib.BspCgResult._fields_}

    def close(self) -> None:
        if self._plan:
            check(lib().bsp_cg_destroy(self._plan))
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# SpMM (replaces smatSpmmfp16, reference src/smat.cu:103; include/smat.h)

def spmm_csr(rowptr, colidx, values, B, C=None, *, alpha: float = 1.0, beta: float = 0.0, stream=None):
    """C = alpha*A*B + beta*C; values/B F16, BF16 or F32; C FP32 (rows x N)."""
    torch = _torch()
    rows = rowptr.numel() - 1
    N = B.shape[1]
    if C is None:
        C = torch.empty(rows, N, dtype=torch.float32, device=B.device)
        beta = 0.0
    if values.dtype != B.dtype:
        raise ValueError("values and B must share a dtype")
    check(lib().bsp_spmm_csr(rows, B.shape[0], colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                             _dptr(values, "values"), _dtype_code(values), _dptr(B, "B"), N, B.stride(0),
                             _dptr(C, "C"), C.stride(0), float(alpha), float(beta), _stream(stream)))
    return C


class SpmmPlan:
    """Row-split plan for CSR SpMM on power-law matrices: rows longer than
    `chunk` nonzeros are cut into chunks handled by separate warps and summed
    in chunk order (deterministic)."""

    def __init__(self, rowptr, colidx, values, *, cols: int, chunk: int = 256, stream=None):
        self._d = _lib.BspSpmmPlan()
        self.rowptr, self.colidx, self.values, self.cols = rowptr, colidx, values, cols
        check(lib().bsp_spmm_plan_create(rowptr.numel() - 1, colidx.numel(), _dptr(rowptr, "rowptr"), chunk,
                                         C.byref(self._d), _stream(stream)))
        self._live = True
        self._ws = None

    @property
    def nchunks(self) -> int:
        return self._d.nchunks

    @property
    def nsplit(self) -> int:
        return self._d.nsplit

    def workspace_bytes(self, N: int) -> int:
        return lib().bsp_spmm_plan_workspace(C.byref(self._d), N)

    @property
    def slab_l2_hints(self) -> int:
        return self._d.slab_l2_hints

    @slab_l2_hints.setter
    def slab_l2_hints(self, v: int) -> None:
        if v not in (0, 1, 2):
            raise ValueError("slab_l2_hints is 0, 1 or 2")
        self._d.slab_l2_hints = v

    _ENGINES = {"auto": 0, "grouped": 1, "slab": 2}

    def spmm(self, B, C_out=None, *, alpha: float = 1.0, beta: float = 0.0, engine: str = "auto",
             slab_cols: int = 0, stream=None):
        """C = alpha*A*B + beta*C.  engine "grouped" (one pass over all
        columns), "slab" (passes over column slabs with length-sorted rows
        spread over lane groups; slab_cols 0 = the default width) or
        "auto"."""
        torch = _torch()
        N = B.shape[1]
        if self.values.dtype != B.dtype:
            raise ValueError("values and B must share a dtype")
        if C_out is None:
            C_out = torch.empty(self._d.rows, N, dtype=torch.float32, device=B.device)
            beta = 0.0
        need = self.workspace_bytes(N)
        if need and (self._ws is None or self._ws.numel() < need):
            self._ws = torch.empty(need, dtype=torch.uint8, device=B.device)
        ws = self._ws if need else None
        check(lib().bsp_spmm_csr_planned_variant(C.byref(self._d), self.cols, self.colidx.numel(),
                                                 _dptr(self.rowptr, "rowptr"), _dptr(self.colidx, "colidx"),
                                                 _dptr(self.values, "values"), _dtype_code(self.values),
                                                 _dptr(B, "B"), N, B.stride(0), _dptr(C_out, "C"), C_out.stride(0),
                                                 float(alpha), float(beta),
                                                 ws.data_ptr() if ws is not None else None, need,
                                                 self._ENGINES[engine], slab_cols, _stream(stream)))
        return C_out

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_spmm_plan_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SmatMatrix:
    """16x16-tile F16/BF16 matrix for the tensor-core (SMaT) SpMM."""

    def __init__(self, rowptr, colidx, values, *, rows: int, cols: int, dtype: str = "f16", stream=None):
        self._d = _lib.BspSmat()
        dt = {"f16": _lib.F16, "bf16": _lib.BF16}[dtype]
        check(lib().bsp_smat_create(rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                    _dptr(values, "values"), dt, C.byref(self._d), _stream(stream)))
        self._live = True

    @property
    def fill(self) -> float:
        return self._d.fill

    @property
    def tiles(self) -> int:
        return self._d.tiles.nonzeroBlocks

    _PATHS = {"auto": 0, "mma_sync": 1, "tcgen05": 2, "tcgen05_w64": 3, "tcgen05_w128": 4, "tcgen05_persistent": 5,
              "tcgen05_persistent_w64": 6}

    def spmm(self, B, C=None, *, alpha: float = 1.0, beta: float = 0.0, path: str = "auto", stream=None):
        """path: "auto" / "tcgen05" (tensor cores, slab width from L2),
        "tcgen05_w64" / "tcgen05_w128" (explicit slab width) or "mma_sync"."""
        torch = _torch()
        N = B.shape[1]
        if C is None:
            C = torch.empty(self._d.rows, N, dtype=torch.float32, device=B.device)
            beta = 0.0
        check(lib().bsp_smat_spmm_path(C_byref(self._d), _dptr(B, "B"), N, B.stride(0), _dptr(C, "C"),
                                       C.stride(0), float(alpha), float(beta), self._PATHS[path], _stream(stream)))
        return C

    def check(self, stream=None) -> None:
        check(lib().bsp_smat_check(C_byref(self._d), _stream(stream)))

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_smat_free(C_byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GatherTileMatrix:
    """Gathered-tile tensor-core SpMM matrix (bsp_gtile) built from host CSR
    arrays: each 16-row group's distinct columns in chunks of 16 with their
    16x16 tiles; C = alpha*A*B + beta*C on tcgen05 with the chunk's B rows
    gathered into shared memory."""

    def __init__(self, A: "HostCSR", dtype: str = "f16"):
        self._d = _lib.BspGtile()
        dt = {"f16": _lib.F16, "bf16": _lib.BF16}[dtype]
        rp = np.ascontiguousarray(A.rowptr, np.int32)
        ci = np.ascontiguousarray(A.colidx, np.int32)
        va = np.ascontiguousarray(A.values, np.float64)
        check(lib().bsp_gtile_create_host(A.rows, A.cols, ci.size, _np_ptr(rp), _np_ptr(ci), _np_ptr(va), dt,
                                          C.byref(self._d)))
        self._live = True
        self._ws = None

    def __getattr__(self, name):
        d = self.__dict__.get("_d")
        if d is not None and name in dict(_lib.BspGtile._fields_):
            return getattr(d, name)
        raise AttributeError(name)

    def chunks_per_group(self) -> np.ndarray:
        d = self._d
        pp = _d2h(d.piece_ptr, d.npieces + 1, np.int32)
        gp = _d2h(d.group_piece, d.ngroups + 1, np.int32)
        return (pp[gp[1:]] - pp[gp[:-1]]).astype(np.int64)

    def spmm(self, B, C_out=None, *, alpha: float = 1.0, beta: float = 0.0, stream=None):
        torch = _torch()
        N = B.shape[1]
        if C_out is None:
            C_out = torch.empty(self._d.rows, N, dtype=torch.float32, device=B.device)
            beta = 0.0
        need = lib().bsp_gtile_workspace(C.byref(self._d), N)
        if need and (self._ws is None or self._ws.numel() < need):
            self._ws = torch.empty(need, dtype=torch.uint8, device=B.device)
        ws = self._ws if need else None
        check(lib().bsp_gtile_spmm(C.byref(self._d), _dptr(B, "B"), N, B.stride(0), _dptr(C_out, "C"),
                                   C_out.stride(0), float(alpha), float(beta),
                                   ws.data_ptr() if ws is not None else None, need, _stream(stream)))
        return C_out

    def check(self, stream=None) -> None:
        check(lib().bsp_gtile_check(C.byref(self._d), _stream(stream)))

    def free(self) -> None:
        if self._live:
            self._live = False
            check(lib().bsp_gtile_free(C.byref(self._d)))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def C_byref(obj):
    return C.byref(obj)


def gen_graph(n: int, alpha: float, mean_deg: float, seed: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_graph, n, alpha, mean_deg, seed)


def gen_banded(n: int, width: int, seed: int) -> HostCSR:
    return _two_phase(lib().bsp_gen_banded, n, width, seed)


# ---------------------------------------------------------------------------
# Batched SpMV / 8-RHS SpMM (no reference counterpart; the reference runs one
# matrix per call, src/csrspmv.cu:104-170)

class BatchPlan:
    """y_m = A_m x_m for many CSR matrices in one persistent, graph-captured
    launch.  `mats` is a list of (rowptr, colidx, values, x, y) device tensors;
    values/x/y F64 or F32; nrhs 1 or 8 (x: cols x 8, y: rows x 8 row-major).
    Matrices with even rows are stored as SELL-32 (sell=False keeps every
    matrix in CSR; sell_wide=True also stores uneven ones as length-sorted
    SELL-32); for the others tune=0 picks lanes per row from row statistics,
    tune=1 times the lane counts per matrix."""

    def __init__(self, mats, *, nrhs: int = 1, tune: int = 0, seg_nnz: int = 512, long_row_nnz: int = 1024,
                 item_nnz: int = 0, use_graph: bool = True, sell: bool = True, sell_wide: bool = False,
                 stream=None):
        torch = _torch()
        if not mats:
            raise ValueError("empty batch")
        dt = mats[0][2].dtype
        if dt not in (torch.float64, torch.float32):
            raise ValueError("batched SpMV takes float64 or float32 values")
        arr = (_lib.BspBatchMat * len(mats))()
        for i, (rp, ci, va, x, y) in enumerate(mats):
            if va.dtype != dt or x.dtype != dt or y.dtype != dt:
                raise ValueError("all values, x and y must share one dtype")
            rows = rp.numel() - 1
            cols = x.shape[0] if nrhs > 1 else x.numel()
            arr[i] = _lib.BspBatchMat(rows, cols, ci.numel(), _dptr(rp, "rowptr"), _dptr(ci, "colidx"),
                                      _dptr(va, "values"), _dptr(x, "x"), _dptr(y, "y"))
        opt = _lib.BspBatchOptions(tune, seg_nnz, long_row_nnz, item_nnz, 1 if use_graph else 0, 1 if sell else 0,
                                   1 if sell_wide else 0)
        self._h = C.c_void_p()
        self.count = len(mats)
        self._keep = list(mats)
        check(lib().bsp_batch_create(len(mats), arr, _lib.F64 if dt == torch.float64 else _lib.F32, nrhs,
                                     C.byref(opt), C.byref(self._h), _stream(stream)))

    def run(self, stream=None) -> None:
        check(lib().bsp_batch_run(self._h, _stream(stream)))

    def run_separate(self, stream=None) -> None:
        check(lib().bsp_batch_run_separate(self._h, _stream(stream)))

    def set_vectors(self, m: int, x, y, stream=None) -> None:
        check(lib().bsp_batch_set_vectors(self._h, m, _dptr(x, "x"), _dptr(y, "y"), _stream(stream)))
        rp, ci, va, _, _ = self._keep[m]
        self._keep[m] = (rp, ci, va, x, y)

    def lanes(self) -> np.ndarray:
        out = np.empty(self.count, np.int32)
        check(lib().bsp_batch_lanes(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def formats(self) -> np.ndarray:
        """Per-matrix storage: 0 = CSR, 1 = SELL-32 (rows in order, 16-bit
        column offsets), 2 = SELL-32 of length-sorted rows (sell_wide=True)."""
        out = np.empty(self.count, np.int32)
        check(lib().bsp_batch_formats(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def stats(self) -> dict:
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().bsp_batch_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"items": a.value, "long_segments": b.value, "nnz": c.value}

    def close(self) -> None:
        if self._h:
            check(lib().bsp_batch_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_batch(count: int, seed: int, n_lo: int = 1000, n_hi: int = 65536) -> list:
    """Seeded batch of matrices: n log-uniform in [n_lo, n_hi]; even entries
    banded (width 3..27), odd entries Zipf(2.2) row lengths capped at n."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        if i % 2 == 0:
            out.append(gen_banded(n, int(rng.integers(3, 28)), seed * 1000 + i))
        else:
            out.append(gen_powerlaw(n, 2.2, n, seed * 1000 + i))
    return out


# ---------------------------------------------------------------------------
# Format autotuner (no reference counterpart)

_FMT_NAMES = {_lib.FMT_CSR: "csr", _lib.FMT_BSR: "bsr", _lib.FMT_DASP: "dasp"}


def _tune_dict(r: "_lib.BspTuneResult") -> dict:
    d = {k: getattr(r, k) for k, _ in _lib.BspTuneResult._fields_}
    d["format_name"] = _FMT_NAMES.get(r.format, "?")
    return d


def tune_spmv(rowptr, colidx, values, *, cols: int, measure: bool = False, stream=None) -> dict:
    """Chooses the FP64 SpMV format for a device CSR matrix (cached by structure)."""
    r = _lib.BspTuneResult()
    check(lib().bsp_tune_spmv(rowptr.numel() - 1, cols, colidx.numel(), _dptr(rowptr, "rowptr"),
                              _dptr(colidx, "colidx"), _dptr(values, "values"), int(measure), C.byref(r),
                              _stream(stream)))
    return _tune_dict(r)


def matrix_key(rowptr, colidx, *, cols: int, stream=None) -> int:
    k = C.c_uint64()
    check(lib().bsp_matrix_key(rowptr.numel() - 1, cols, colidx.numel(), _dptr(rowptr, "rowptr"),
                               _dptr(colidx, "colidx"), C.byref(k), _stream(stream)))
    return k.value


def tune_cache_clear() -> None:
    lib().bsp_tune_cache_clear()


class SpmvPlan:
    """Tuned FP64 SpMV: converts once to the chosen format and runs it (the
    CSR tensors must stay alive)."""

    def __init__(self, rowptr, colidx, values, *, cols: int, measure: bool = False, stream=None):
        self._keep = (rowptr, colidx, values)
        self.rows = rowptr.numel() - 1
        self._h = C.c_void_p()
        check(lib().bsp_spmv_plan_create(self.rows, cols, colidx.numel(), _dptr(rowptr, "rowptr"),
                                         _dptr(colidx, "colidx"), _dptr(values, "values"), int(measure),
                                         C.byref(self._h), _stream(stream)))

    @property
    def choice(self) -> dict:
        r = _lib.BspTuneResult()
        check(lib().bsp_spmv_plan_choice(self._h, C.byref(r)))
        return _tune_dict(r)

    def spmv(self, x, y=None, *, alpha: float = 1.0, beta: float = 0.0, stream=None):
        torch = _torch()
        if y is None:
            y = torch.empty(self.rows, dtype=torch.float64, device=x.device)
            beta = 0.0
        check(lib().bsp_spmv_plan_run(self._h, _dptr(x, "x"), _dptr(y, "y"), float(alpha), float(beta),
                                      _stream(stream)))
        return y

    def close(self) -> None:
        if self._h:
            check(lib().bsp_spmv_plan_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Reordering (no reference counterpart)

def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def reorder_rcm_host(rowptr: np.ndarray, colidx: np.ndarray) -> np.ndarray:
    """Reverse Cuthill-McKee permutation (perm[new] = old) of host CSR arrays."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    perm = np.empty(rowptr.size - 1, np.int32)
    check(lib().bsp_reorder_rcm_host(perm.size, colidx.size, _np_ptr(rowptr), _np_ptr(colidx), _np_ptr(perm)))
    return perm


def permute_csr_host(A: "HostCSR", perm: np.ndarray) -> "HostCSR":
    """P A P^T of a square host CSR matrix."""
    perm = np.ascontiguousarray(perm, np.int32)
    rp = np.empty(A.rows + 1, np.int32)
    ci = np.empty(A.nnz, np.int32)
    va = np.empty(A.nnz, np.float64)
    check(lib().bsp_permute_csr_host(A.rows, A.nnz, _np_ptr(np.ascontiguousarray(A.rowptr, np.int32)),
                                     _np_ptr(np.ascontiguousarray(A.colidx, np.int32)),
                                     _np_ptr(np.ascontiguousarray(A.values, np.float64)), _np_ptr(perm),
                                     _np_ptr(rp), _np_ptr(ci), _np_ptr(va)))
    return HostCSR(A.rows, A.cols, rp, ci, va)


def reorder_rcm(rowptr, colidx, stream=None):
    """Device form: returns perm as an int32 tensor on the same device."""
    torch = _torch()
    perm = torch.empty(rowptr.numel() - 1, dtype=torch.int32, device=rowptr.device)
    check(lib().bsp_reorder_rcm(perm.numel(), colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                _dptr(perm, "perm"), _stream(stream)))
    return perm


def reorder_similarity_host(rowptr: np.ndarray, colidx: np.ndarray, cols: int, group_rows: int = 16,
                            block_cols: int = 16) -> np.ndarray:
    """Row-similarity permutation (perm[new] = old) of host CSR arrays: rows
    with similar column-block sets land in the same group of group_rows."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    perm = np.empty(rowptr.size - 1, np.int32)
    check(lib().bsp_reorder_similarity_host(perm.size, cols, colidx.size, _np_ptr(rowptr), _np_ptr(colidx),
                                            group_rows, block_cols, _np_ptr(perm)))
    return perm


def permute_rows_csr_host(A: "HostCSR", perm: np.ndarray) -> "HostCSR":
    """P A (rows only) of a host CSR matrix."""
    perm = np.ascontiguousarray(perm, np.int32)
    rp = np.empty(A.rows + 1, np.int32)
    ci = np.empty(A.nnz, np.int32)
    va = np.empty(A.nnz, np.float64)
    check(lib().bsp_permute_rows_csr_host(A.rows, A.nnz, _np_ptr(np.ascontiguousarray(A.rowptr, np.int32)),
                                          _np_ptr(np.ascontiguousarray(A.colidx, np.int32)),
                                          _np_ptr(np.ascontiguousarray(A.values, np.float64)), _np_ptr(perm),
                                          _np_ptr(rp), _np_ptr(ci), _np_ptr(va)))
    return HostCSR(A.rows, A.cols, rp, ci, va)


def choose_spmm_host(A: "HostCSR", N: int, reorder: bool = True) -> tuple:
    """SpMM engine for C = A B with N columns of B: ({engine: "smat",
    "gtile" or "csr", smat_path, reorder, tile and chunk counts, time
    estimates}, perm or None).  With reorder, perm is the row-similarity
    order (apply it with permute_rows_csr_host when the choice says
    reorder)."""
    rp = np.ascontiguousarray(A.rowptr, np.int32)
    ci = np.ascontiguousarray(A.colidx, np.int32)
    perm = np.empty(A.rows, np.int32) if reorder else None
    c = _lib.BspSpmmChoice()
    check(lib().bsp_spmm_choose_host(A.rows, A.cols, ci.size, _np_ptr(rp), _np_ptr(ci), N,
                                     _np_ptr(perm) if perm is not None else None, C.byref(c)))
    d = {k: getattr(c, k) for k, _ in _lib.BspSpmmChoice._fields_ if k != "reserved"}
    d["engine"] = {_lib.BSP_SPMM_ENGINE_SMAT: "smat", _lib.BSP_SPMM_ENGINE_GTILE: "gtile"}.get(c.engine, "csr")
    d["smat_path"] = {v: k for k, v in SmatMatrix._PATHS.items()}[c.smat_path]
    d["reorder"] = bool(c.reorder)
    return d, perm


def reorder_similarity(rowptr, colidx, cols: int, group_rows: int = 16, block_cols: int = 16, stream=None):
    """Device form of reorder_similarity_host: perm as an int32 tensor."""
    torch = _torch()
    perm = torch.empty(rowptr.numel() - 1, dtype=torch.int32, device=rowptr.device)
    check(lib().bsp_reorder_similarity(perm.numel(), cols, colidx.numel(), _dptr(rowptr, "rowptr"),
                                       _dptr(colidx, "colidx"), group_rows, block_cols, _dptr(perm, "perm"),
                                       _stream(stream)))
    return perm


def permute_rows_csr(rowptr, colidx, values, perm, stream=None):
    """Device form of P A (rows only); returns (rowptr, colidx, values)."""
    torch = _torch()
    rp = torch.empty_like(rowptr)
    ci = torch.empty_like(colidx)
    va = torch.empty_like(values)
    check(lib().bsp_permute_rows_csr(perm.numel(), colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                     _dptr(values, "values"), _dptr(perm, "perm"), _dptr(rp, "out_rowptr"),
                                     _dptr(ci, "out_colidx"), _dptr(va, "out_values"), _stream(stream)))
    return rp, ci, va


def permute_csr(rowptr, colidx, values, perm, stream=None):
    """Device form of P A P^T; returns (rowptr, colidx, values) tensors."""
    torch = _torch()
    rp = torch.empty_like(rowptr)
    ci = torch.empty_like(colidx)
    va = torch.empty_like(values)
    check(lib().bsp_permute_csr(perm.numel(), colidx.numel(), _dptr(rowptr, "rowptr"), _dptr(colidx, "colidx"),
                                _dptr(values, "values"), _dptr(perm, "perm"), _dptr(rp, "out_rowptr"),
                                _dptr(ci, "out_colidx"), _dptr(va, "out_values"), _stream(stream)))
    return rp, ci, va



# ---------------------------------------------------------------------------
# Matrix Market files (replaces the drivers' read_triplet_file + triplet sort,
# reference bench/spmvfp64.cpp:37-86)

_MTX_FORMATS = {0: "coordinate", 1: "array"}
_MTX_FIELDS = {0: "real", 1: "integer", 2: "pattern"}
_MTX_SYMMETRIES = {0: "general", 1: "symmetric", 2: "skew-symmetric", 3: "hermitian"}


class MtxFile:
    """A parsed Matrix Market file (host triplets held by the library).

    ``fmm_diag_zero`` adds an explicit 0.0 mirror for every diagonal entry of
    a non-general file, fast_matrix_market's default element count."""

    def __init__(self, path, *, fmm_diag_zero: bool = False, flags: int = 0, threads: int = 0):
        h = C.c_void_p()
        flags = int(flags) | (_lib.MTX_DIAG_ZERO if fmm_diag_zero else 0)
        check(lib().bsp_mtx_read(os.fsencode(os.fspath(path)), flags, int(threads), C.byref(h)))
        self._h = h
        info = _lib.BspMtxInfo()
        check(lib().bsp_mtx_get_info(h, C.byref(info)))
        self.rows, self.cols, self.entries, self.nnz = info.rows, info.cols, info.entries, info.nnz
        self.format = _MTX_FORMATS[info.format]
        self.field = _MTX_FIELDS[info.field]
        self.symmetry = _MTX_SYMMETRIES[info.symmetry]

    def triplets(self) -> tuple:
        r = np.empty(self.nnz, np.int32)
        c = np.empty(self.nnz, np.int32)
        v = np.empty(self.nnz, np.float64)
        check(lib().bsp_mtx_triplets(self._h, _np_ptr(r), _np_ptr(c), _np_ptr(v)))
        return r, c, v

    def csr_host(self) -> HostCSR:
        rp = np.empty(self.rows + 1, np.int32)
        ci = np.empty(self.nnz, np.int32)
        va = np.empty(self.nnz, np.float64)
        check(lib().bsp_mtx_csr_host(self._h, _np_ptr(rp), _np_ptr(ci), _np_ptr(va)))
        return HostCSR(int(self.rows), int(self.cols), rp, ci, va)

    def csr(self, device="cuda", stream=None) -> tuple:
        """CSR built on the device: (rowptr, colidx, values) tensors."""
        torch = _torch()
        rp = torch.empty(self.rows + 1, dtype=torch.int32, device=device)
        ci = torch.empty(max(1, self.nnz), dtype=torch.int32, device=device)
        va = torch.empty(max(1, self.nnz), dtype=torch.float64, device=device)
        check(lib().bsp_mtx_csr(self._h, _dptr(rp, "rowptr"), _dptr(ci, "colidx"), _dptr(va, "values"),
                                _stream(stream)))
        return rp, ci[:self.nnz], va[:self.nnz]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().bsp_mtx_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_mtx(path, *, fmm_diag_zero: bool = False, threads: int = 0) -> HostCSR:
    """Host CSR of a Matrix Market file (rows, then columns ascending)."""
    f = MtxFile(path, fmm_diag_zero=fmm_diag_zero, threads=threads)
    try:
        return f.csr_host()
    finally:
        f.close()


def write_mtx(path, A: HostCSR, *, pattern: bool = False, threads: int = 0) -> None:
    """Writes host CSR as 'coordinate real general' (shortest round-trip values)."""
    rp = np.ascontiguousarray(A.rowptr, np.int32)
    ci = np.ascontiguousarray(A.colidx, np.int32)
    va = None if pattern else np.ascontiguousarray(A.values, np.float64)
    check(lib().bsp_mtx_write_csr_host(os.fsencode(os.fspath(path)), A.rows, A.cols, ci.size, _np_ptr(rp),
                                       _np_ptr(ci), None if va is None else _np_ptr(va), int(threads)))


def gather_probe(buf, width: int, count: int, seed: int = 1, stream=None) -> None:
    """Launches the random-gather rate probe over the device tensor `buf`
    (`count` gathers of `width` bytes); time it with CUDA events."""
    torch = _torch()
    sink = torch.zeros(1, dtype=torch.int64, device=buf.device)
    check(lib().bsp_gather_probe(_dptr(buf, "buf"), buf.numel() * buf.element_size(), width, count, seed,
                                 _dptr(sink, "sink"), _stream(stream)))
