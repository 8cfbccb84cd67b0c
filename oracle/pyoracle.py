"""ctypes loader for the CPU oracle (liboracle.so) and, when built, the
reference's own code (oracle/_ref).  TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the library never imports it.
"""
from __future__ import annotations

import ctypes as C
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64


def _p(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


_orc = None


def build() -> None:
    """Builds liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build()
        L = C.CDLL(str(ORACLE_SO))
        L.orc_spmv_f64.argtypes = [_I64, _P, _P, _P, _P, _P]
        L.orc_spmv_f64_i32.argtypes = [_I32, _P, _P, _P, _P, _P]
        L.orc_spmv_f32.argtypes = [_I32, _P, _P, _P, _P, _P]
        L.orc_spmv_f16.argtypes = [_I32, _P, _P, _P, _P, _P]
        L.orc_abs_rowsum.argtypes = [_I32, _P, _P, _P, _P, _P]
        L.orc_spmm_f64.argtypes = [_I32, _P, _P, _P, _I32, _P, _P, _P]
        L.orc_csr2bsr.restype = _I64
        L.orc_csr2bsr.argtypes = [_I32, _I32, _P, _P, _P, _I32, _P, _P, _P, _P]
        L.orc_bsr_chunks.restype = _I32
        L.orc_bsr_chunks.argtypes = [_I32, _P, _P, _P]
        L.orc_bsr_stand.restype = C.c_double
        L.orc_bsr_stand.argtypes = [_I32, _P]
        L.orc_recorder.argtypes = [_I32, _P, _P, _P, _P, _P, _P, _P]
        L.orc_dbsr_blocks.restype = _I32
        L.orc_dbsr_blocks.argtypes = [_I32, _P, _P]
        L.orc_dbsr_fill.argtypes = [_I32, _P, _P, _P, _P, _P, _P, _P]
        L.orc_dbsr_balance.restype = _I32
        L.orc_dbsr_balance.argtypes = [_I32, _P, _P, _I32, _P]
        L.orc_csr2bcsr.restype = _I64
        L.orc_csr2bcsr.argtypes = [_I32, _I32, _P, _P, _P, _I32, _I32, _P, _P, _P, _P]
        L.orc_f32_to_f16.restype = C.c_uint16
        L.orc_f32_to_f16.argtypes = [C.c_float]
        _orc = L
    return _orc


# ---------------------------------------------------------------------------
# SpMV (src/ref.cpp)

def spmv_f64(rowptr, colidx, val, x) -> np.ndarray:
    rows = rowptr.size - 1
    y = np.empty(rows, np.float64)
    orc().orc_spmv_f64_i32(rows, _p(rowptr), _p(colidx), _p(val), _p(x), _p(y))
    return y


def spmv_f32(rowptr, colidx, val, x) -> np.ndarray:
    rows = rowptr.size - 1
    y = np.empty(rows, np.float32)
    orc().orc_spmv_f32(rows, _p(rowptr), _p(colidx), _p(np.ascontiguousarray(val, np.float32)),
                       _p(np.ascontiguousarray(x, np.float32)), _p(y))
    return y


def spmv_f16(rowptr, colidx, val16: np.ndarray, x16: np.ndarray) -> np.ndarray:
    """val16/x16 are float16 arrays; returns float16."""
    rows = rowptr.size - 1
    y = np.empty(rows, np.uint16)
    orc().orc_spmv_f16(rows, _p(rowptr), _p(colidx), _p(val16.view(np.uint16)), _p(x16.view(np.uint16)), _p(y))
    return y.view(np.float16)


def abs_rowsum(rowptr, colidx, val, x) -> np.ndarray:
    rows = rowptr.size - 1
    y = np.empty(rows, np.float64)
    orc().orc_abs_rowsum(rows, _p(rowptr), _p(colidx), _p(val), _p(x), _p(y))
    return y


def spmm_f64(rowptr, colidx, val, B):
    """FP64 C = A*B and |A|*|B| (for the error bound)."""
    rows = rowptr.size - 1
    B = np.ascontiguousarray(B, np.float64)
    N = B.shape[1]
    Cm = np.empty((rows, N), np.float64)
    absC = np.empty((rows, N), np.float64)
    orc().orc_spmm_f64(rows, _p(np.ascontiguousarray(rowptr, np.int32)), _p(np.ascontiguousarray(colidx, np.int32)),
                       _p(np.ascontiguousarray(val, np.float64)), N, _p(B), _p(Cm), _p(absC))
    return Cm, absC


def spmv_tolerance(rowptr, colidx, val, x, unit: float = 2.0 ** -53) -> np.ndarray:
    """Per-row bound on |y_gpu - y_oracle| for any summation order:
    2 * gamma_L * sum_j |a_ij x_j| with gamma_L = L*u/(1-L*u), L = row length
    + 1 (both results carry at most gamma_L relative error)."""
    L = np.diff(rowptr).astype(np.float64) + 1.0
    g = L * unit / (1.0 - L * unit)
    return 2.0 * g * abs_rowsum(rowptr, colidx, val, x) + np.finfo(np.float64).tiny


# ---------------------------------------------------------------------------
# AmgT BSR (src/amgT.cu:1114-1200)

def csr2bsr(rows, cols, rowptr, colidx, val, bs=4) -> dict:
    L = orc()
    nb = int(L.orc_csr2bsr(rows, cols, _p(rowptr), _p(colidx), _p(val), bs, None, None, None, None))
    brow = (rows + bs - 1) // bs
    blcPtr = np.empty(brow + 1, np.int32)
    blcIdx = np.empty(nb, np.int32)
    blcVal = np.empty(nb * bs * bs, np.float64)
    blcMap = np.empty(nb, np.uint64)
    L.orc_csr2bsr(rows, cols, _p(rowptr), _p(colidx), _p(val), bs, _p(blcPtr), _p(blcIdx), _p(blcVal), _p(blcMap))
    warpnum = int(L.orc_bsr_chunks(brow, _p(blcPtr), None, None))
    rpw = np.empty(brow + 1, np.int32)
    riw = np.empty(warpnum, np.int32)
    L.orc_bsr_chunks(brow, _p(blcPtr), _p(rpw), _p(riw))
    return {"blc_row": brow, "blc_num": nb, "blcPtr": blcPtr, "blcIdx": blcIdx, "blcVal": blcVal,
            "blcMap": blcMap.astype(np.uint16) if bs == 4 else blcMap, "rowPtrbyWarp": rpw,
            "rowIdxbyWarp": riw, "warpnum": warpnum, "stand": float(L.orc_bsr_stand(brow, _p(blcPtr))),
            "avg_nnz": (colidx.size / nb) if nb else 0.0}


# ---------------------------------------------------------------------------
# DBSR (include/dbsr.h) and BCSR (utils/utils.hpp)

def recorder(rowptr, colidx, val) -> dict:
    rows = rowptr.size - 1
    order = np.empty(rows, np.int32)
    rp = np.empty(rows + 1, np.int32)
    ci = np.empty(colidx.size, np.int32)
    va = np.empty(colidx.size, np.float64)
    orc().orc_recorder(rows, _p(rowptr), _p(colidx), _p(val), _p(order), _p(rp), _p(ci), _p(va))
    return {"order": order, "rowptr": rp, "colidx": ci, "values": va}


def csr2dbsr(rowptr, colidx, val, recorder_sort: bool) -> dict:
    L = orc()
    rows = rowptr.size - 1
    out = {}
    if recorder_sort:
        rec = recorder(rowptr, colidx, val)
        rowptr, colidx, val = rec["rowptr"], rec["colidx"], rec["values"]
        out["recorderMap"] = rec["order"]
        out["rec_rowptr"], out["rec_colidx"], out["rec_values"] = rowptr, colidx, val
    brow = (rows + 3) // 4
    blcPtr = np.empty(brow + 1, np.int32)
    nb = int(L.orc_dbsr_blocks(rows, _p(rowptr), _p(blcPtr)))
    col = np.zeros(nb * 16, np.int32)
    bv = np.zeros(nb * 16, np.float64)
    mp = np.zeros(max(nb, 1), np.uint16)
    L.orc_dbsr_fill(rows, _p(rowptr), _p(colidx), _p(val), _p(blcPtr), _p(col), _p(bv), _p(mp))
    of = C.c_int32()
    wn = int(L.orc_dbsr_balance(brow, _p(blcPtr), None, 0, C.byref(of)))
    prefix = np.empty(wn + 1, np.int32)
    L.orc_dbsr_balance(brow, _p(blcPtr), _p(prefix), wn, C.byref(of))
    out.update(blc_row=brow, blc_num=nb, blocknnz=nb * 16, blcPtr=blcPtr, colIdx=col, blcVal=bv, blcMap=mp[:nb],
               warpnum=wn, prefix=prefix, balance_overflow=int(of.value))
    return out


def csr2bcsr(rows, cols, rowptr, colidx, val, tm, tk, with_mapping=True) -> dict:
    L = orc()
    nb = int(L.orc_csr2bcsr(rows, cols, _p(rowptr), _p(colidx), _p(val), tm, tk, None, None, None, None))
    nr = (rows + tm - 1) // tm
    nc = (cols + tk - 1) // tk
    rp = np.empty(nr + 1, np.int32)
    ci = np.empty(nb, np.int32)
    bv = np.empty(nb * tm * tk, np.float64)
    mp = np.empty(nr * nc, np.int32) if with_mapping else None
    L.orc_csr2bcsr(rows, cols, _p(rowptr), _p(colidx), _p(val), tm, tk, _p(rp), _p(ci), _p(bv),
                   _p(mp) if mp is not None else None)
    return {"rowRegions": nr, "colRegions": nc, "nonzeroBlocks": nb, "bcsrRowPtr": rp, "bcsrColIdx": ci,
            "bcsrVal": bv, "mapping": mp}


# ---------------------------------------------------------------------------
# The reference's own code (oracle/_ref), when built

def ref_available() -> bool:
    return (REF_DIR / "libref_host.so").exists()


def write_csr_bin(path, rows, cols, rowptr, colidx, val, x, threshold=0.75, block_longest=256) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<iiidi", rows, cols, int(colidx.size), float(threshold), int(block_longest)))
        f.write(np.ascontiguousarray(rowptr, np.int32).tobytes())
        f.write(np.ascontiguousarray(colidx, np.int32).tobytes())
        f.write(np.ascontiguousarray(val, np.float64).tobytes())
        f.write(np.ascontiguousarray(x, np.float64).tobytes())


def read_records(path) -> dict:
    d = Path(path).read_bytes()
    o = 0
    out = {}
    while o < len(d):
        (nl,) = struct.unpack_from("<i", d, o)
        o += 4
        name = d[o:o + nl].decode()
        o += nl
        (nb,) = struct.unpack_from("<q", d, o)
        o += 8
        out[name] = d[o:o + nb]
        o += nb
    return out


def run_capture(exe: str, rows, cols, rowptr, colidx, val, x, threshold=0.75, block_longest=256) -> dict:
    """Runs oracle/_ref/<exe> (dasp_capture or amgt_capture) on a CSR matrix."""
    with tempfile.TemporaryDirectory() as td:
        fin = Path(td) / "in.bin"
        fout = Path(td) / "out.bin"
        write_csr_bin(fin, rows, cols, rowptr, colidx, val, x, threshold, block_longest)
        r = subprocess.run([str(REF_DIR / exe), str(fin), str(fout)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{exe} failed ({r.returncode}): {r.stdout[-2000:]} {r.stderr[-2000:]}")
        return read_records(fout)


# ---------------------------------------------------------------------------
# DASP packing (src/dasp.cu:827-1482)

_DASP_INTS = ["row_long", "row_block", "row_zero", "short_row_1", "short_row_2", "short_row_3", "short_row_4",
              "common_13", "short_row_34", "fill0_nnz_short13", "fill0_nnz_short34", "fill0_nnz_short",
              "fill0_nnz_long", "blocknum", "fill0_nnz_reg", "nnz_irreg", "offset_reg", "offset_short1",
              "offset_short13", "offset_short34", "offset_short22", "block_num_all"]


class _OrcDasp(C.Structure):
    _fields_ = [(n, C.c_int32) for n in _DASP_INTS] + [
        ("short_val", C.POINTER(C.c_double)), ("long_val", C.POINTER(C.c_double)),
        ("reg_val", C.POINTER(C.c_double)), ("irreg_val", C.POINTER(C.c_double)),
        ("short_cid", C.POINTER(C.c_int32)), ("long_cid", C.POINTER(C.c_int32)),
        ("long_ptr_warp", C.POINTER(C.c_int32)), ("reg_cid", C.POINTER(C.c_int32)),
        ("block_ptr", C.POINTER(C.c_int32)), ("irreg_cid", C.POINTER(C.c_int32)),
        ("irreg_rpt", C.POINTER(C.c_int32)), ("order_rid", C.POINTER(C.c_int32))]


def dasp_pack(rowptr, colidx, val, threshold=0.75, block_longest=256) -> dict:
    L = orc()
    L.orc_dasp_pack.argtypes = [_I32, _P, _P, _P, C.c_double, _I32, C.POINTER(_OrcDasp)]
    L.orc_dasp_free.argtypes = [C.POINTER(_OrcDasp)]
    o = _OrcDasp()
    rows = rowptr.size - 1
    L.orc_dasp_pack(rows, _p(rowptr), _p(colidx), _p(val), float(threshold), int(block_longest), C.byref(o))

    def arr(ptr, n, dt):
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).copy() if n > 0 else np.zeros(0, dt)

    out = {n: int(getattr(o, n)) for n in _DASP_INTS}
    lw = o.long_ptr_warp[o.row_long]
    out.update(
        short_val=arr(o.short_val, o.fill0_nnz_short, np.float64), short_cid=arr(o.short_cid, o.fill0_nnz_short, np.int32),
        long_val=arr(o.long_val, o.fill0_nnz_long, np.float64), long_cid=arr(o.long_cid, o.fill0_nnz_long, np.int32),
        long_ptr_warp=arr(o.long_ptr_warp, o.row_long + 1, np.int32),
        reg_val=arr(o.reg_val, o.fill0_nnz_reg, np.float64), reg_cid=arr(o.reg_cid, o.fill0_nnz_reg, np.int32),
        block_ptr=arr(o.block_ptr, o.blocknum + 1, np.int32),
        irreg_val=arr(o.irreg_val, o.nnz_irreg, np.float64), irreg_cid=arr(o.irreg_cid, o.nnz_irreg, np.int32),
        irreg_rpt=arr(o.irreg_rpt, o.row_block + 1, np.int32), order_rid=arr(o.order_rid, rows, np.int32),
        long_warps=int(lw))
    L.orc_dasp_free(C.byref(o))
    return out


# ---------------------------------------------------------------------------
# Block statistics (bench/blockinfo.cpp:96-119)

def blockinfo(rowptr, colidx) -> dict:
    L = orc()
    L.orc_blockinfo.argtypes = [_I32, _P, _P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    b, br = C.c_int64(), C.c_int64()
    L.orc_blockinfo(rowptr.size - 1, _p(rowptr), _p(colidx), C.byref(b), C.byref(br))
    return {"blocks": b.value, "blocks_recorder": br.value}


def write_mtx(path, rows, cols, rowptr, colidx, values) -> None:
    """Matrix Market coordinate file (1-based, general, real)."""
    r = np.repeat(np.arange(rows, dtype=np.int64), np.diff(rowptr)) + 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{rows} {cols} {colidx.size}\n")
        np.savetxt(f, np.column_stack([r, colidx.astype(np.int64) + 1, values]), fmt="%d %d %.17g")


def run_ref_blockinfo(rows, cols, rowptr, colidx, values) -> dict:
    """The reference's bench/blockinfo.cpp (oracle/_ref/blockinfo) on a matrix."""
    import re
    with tempfile.TemporaryDirectory() as td:
        p = Path(td) / "m.mtx"
        write_mtx(p, rows, cols, rowptr, colidx, values)
        out = subprocess.run([str(REF_DIR / "blockinfo"), str(p)], capture_output=True, text=True, check=True).stdout
    nums = re.findall(r"block num:(\d+)", out)
    return {"blocks": int(nums[0]), "blocks_recorder": int(nums[1])}


def cg(rowptr, colidx, val, b, tol=1e-10, max_iters=100000) -> tuple:
    """FP64 CG on the CPU (x0 = 0); returns (x, iterations)."""
    L = orc()
    L.orc_cg.restype = _I32
    L.orc_cg.argtypes = [_I32, _P, _P, _P, _P, _P, C.c_double, _I32]
    n = rowptr.size - 1
    x = np.zeros(n)
    it = L.orc_cg(n, _p(rowptr), _p(colidx), _p(val), _p(np.ascontiguousarray(b, np.float64)), _p(x), tol, max_iters)
    return x, int(it)


def pcg(rowptr, colidx, val, b, bs, tol=1e-10, max_iters=100000) -> tuple:
    """FP64 block-Jacobi PCG on the CPU (bs = 1: Jacobi; x0 = 0); returns
    (x, iterations)."""
    L = orc()
    L.orc_pcg.restype = _I32
    L.orc_pcg.argtypes = [_I32, _P, _P, _P, _P, _P, C.c_double, _I32, _I32]
    n = rowptr.size - 1
    x = np.zeros(n)
    it = L.orc_pcg(n, _p(rowptr), _p(colidx), _p(val), _p(np.ascontiguousarray(b, np.float64)), _p(x), tol,
                   max_iters, bs)
    return x, int(it)


def block_jacobi(rowptr, colidx, val, bs) -> np.ndarray:
    """Inverted diagonal blocks of bs rows, [nblocks, bs, bs] (None if singular)."""
    L = orc()
    L.orc_block_jacobi.restype = _I32
    L.orc_block_jacobi.argtypes = [_I32, _P, _P, _P, _I32, _P]
    n = rowptr.size - 1
    nb = (n + bs - 1) // bs
    out = np.zeros((nb, bs, bs))
    rc = L.orc_block_jacobi(n, _p(rowptr), _p(colidx), _p(val), bs, _p(out))
    return None if rc != 0 else out


def rel_residual(rowptr, colidx, val, b, x) -> float:
    """||b - A x|| / ||b|| with the oracle SpMV."""
    r = b - spmv_f64(rowptr, colidx, val, np.ascontiguousarray(x, np.float64))
    return float(np.linalg.norm(r) / np.linalg.norm(b))


# ---------------------------------------------------------------------------
# Benchmark inputs without the library (oracle_gen.c)

def gen_stencil27(m: int, dof: int, seed: int) -> tuple:
    """The seeded 27-point stencil (m^3 nodes x dof) as (rowptr, colidx,
    values), bit-identical to the library's generator."""
    L = orc()
    L.orc_gen_stencil27.restype = _I64
    L.orc_gen_stencil27.argtypes = [_I32, _I32, C.c_uint64, _P, _P, _P]
    n = m * m * m * dof
    rowptr = np.empty(n + 1, np.int32)
    nnz = int(L.orc_gen_stencil27(m, dof, seed, _p(rowptr), None, None))
    if nnz < 0:
        raise ValueError("stencil too large for int32 indices")
    colidx = np.empty(nnz, np.int32)
    values = np.empty(nnz, np.float64)
    L.orc_gen_stencil27(m, dof, seed, _p(rowptr), _p(colidx), _p(values))
    return rowptr, colidx, values


def gen_uniform(n: int, seed: int) -> np.ndarray:
    """The seeded uniform [-1, 1) vector, bit-identical to the library's."""
    L = orc()
    L.orc_gen_uniform.restype = None
    L.orc_gen_uniform.argtypes = [_I64, C.c_uint64, _P]
    x = np.empty(n, np.float64)
    L.orc_gen_uniform(n, seed, _p(x))
    return x


# ---------------------------------------------------------------------------
# Per-block power-of-two-scaled FP16/BF16 BSR (oracle_formats.c)

def bsr_scale(blcIdx, blcVal, bs: int, dtype: str) -> tuple:
    """(key, val, bad) of the library's scaled BSR format from FP64 blocks."""
    L = orc()
    L.orc_bsr_scale.restype = _I32
    L.orc_bsr_scale.argtypes = [_I64, _I32, _I32, _P, _P, _P, _P]
    nb = blcIdx.size
    key = np.empty(nb, np.uint32)
    val = np.empty(nb * bs * bs, np.uint16)
    dt = {"f16": 2, "bf16": 3}[dtype]
    bad = L.orc_bsr_scale(nb, bs, dt, _p(np.ascontiguousarray(blcIdx, np.int32)),
                          _p(np.ascontiguousarray(blcVal, np.float64)), _p(key), _p(val))
    return key, val, int(bad)


def bsr_unscale(key, val, bs: int, dtype: str) -> np.ndarray:
    """Exact FP64 values of scaled blocks, row-major per block."""
    L = orc()
    L.orc_bsr_unscale.restype = None
    L.orc_bsr_unscale.argtypes = [_I64, _I32, _I32, _P, _P, _P]
    out = np.empty(val.size, np.float64)
    L.orc_bsr_unscale(key.size, bs, {"f16": 2, "bf16": 3}[dtype], _p(key), _p(val), _p(out))
    return out


def bsr_spmv_f64(rows: int, blcPtr, blcIdx, blockvals, bs: int, x) -> tuple:
    """FP64 y = A x of a BSR matrix given by row-major FP64 blocks, and
    sum_j |a_ij x_j| per row (for the rounding bound); x is zero-padded to
    whole block columns."""
    nb = blcIdx.size
    brow = blcPtr.size - 1
    V = np.asarray(blockvals, np.float64).reshape(nb, bs, bs)
    xp = np.zeros(((x.size + bs - 1) // bs + 1) * bs)
    xp[:x.size] = x
    Xb = xp[blcIdx.astype(np.int64)[:, None] * bs + np.arange(bs)[None, :]]          # [nb, bs]
    part = np.einsum("krc,kc->kr", V, Xb)
    apart = np.einsum("krc,kc->kr", np.abs(V), np.abs(Xb))
    owner = np.repeat(np.arange(brow), np.diff(blcPtr))
    y = np.zeros((brow, bs))
    ay = np.zeros((brow, bs))
    np.add.at(y, owner, part) if nb < 4096 else _segsum(y, blcPtr, part)
    np.add.at(ay, owner, apart) if nb < 4096 else _segsum(ay, blcPtr, apart)
    return y.reshape(-1)[:rows], ay.reshape(-1)[:rows]


def _segsum(out, ptr, part) -> None:
    """out[b] = sum of part[ptr[b]:ptr[b+1]] (rows of 2-D arrays)."""
    nz = np.flatnonzero(np.diff(ptr) > 0)
    if nz.size:
        out[nz] = np.add.reduceat(part, ptr[nz].astype(np.int64), axis=0)
