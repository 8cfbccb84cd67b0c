"""Generates the golden fixtures in tests/golden/ by running the reference's
own code, compiled from its sources into oracle/_ref (see oracle/Makefile):

  spmv_*.npz   ref_spmv_fp64 / ref_spmv_fp32 / ref_spmv_fp16 (src/ref.cpp)
  bcsr_*.npz   csrToBcsr (utils/utils.hpp:10)
  dbsr_*.npz   csrTodbsrWithRecorder and csrTodbsr + balanceDbsr (include/dbsr.h)
  dasp_*.npz   every array spmv_all (src/dasp.cu:814) uploads, captured on the
               CPU through oracle/cuda_host_stub.cpp
  amgt_*.npz   CSR2BSR_GPU + BSR_BALANCED_PREPROCESS_GPU (src/amgT.cu:1114),
               only with --amgt on a machine with a GPU

Inputs are small seeded matrices (numpy PCG64), stored in the fixtures.

    python tests/golden/make_golden.py           # needs the reference tree
    python tests/golden/make_golden.py --amgt    # adds the AmgT fixtures (GPU)
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import pyoracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def matrices() -> dict:
    """Small seeded CSR inputs covering the row classes the paths care about."""
    mats = {}
    rng = np.random.default_rng(20261203)

    def from_rows(n_rows, n_cols, cols_per_row, vals=None):
        rp = np.zeros(n_rows + 1, np.int32)
        rp[1:] = np.cumsum([len(c) for c in cols_per_row])
        ci = np.concatenate([np.asarray(c, np.int32) for c in cols_per_row]) if rp[-1] else np.zeros(0, np.int32)
        va = rng.standard_normal(ci.size) if vals is None else vals
        return dict(rows=n_rows, cols=n_cols, rowptr=rp, colidx=ci, values=va.astype(np.float64))

    # 2-D 5-point Laplacian 16x16
    nx = 16
    rows = []
    vals = []
    for i in range(nx * nx):
        x, y = i % nx, i // nx
        c = []
        v = []
        if y > 0:
            c.append(i - nx); v.append(-1.0)
        if x > 0:
            c.append(i - 1); v.append(-1.0)
        c.append(i); v.append(4.0)
        if x < nx - 1:
            c.append(i + 1); v.append(-1.0)
        if y < nx - 1:
            c.append(i + nx); v.append(-1.0)
        rows.append(c)
        vals.extend(v)
    mats["lap16"] = from_rows(nx * nx, nx * nx, rows, np.array(vals))

    # power-law rows (Zipf 2.0, capped), every DASP row class present
    n = 2000
    lens = np.minimum(rng.zipf(2.0, n), 400)
    lens[::97] = 0  # some empty rows
    mats["powerlaw2k"] = from_rows(n, n, [np.sort(rng.choice(n, int(l), replace=False)) for l in lens])

    # random block-sparse: 64 block-rows of 4x4, 6 block columns each, random fill
    nbr, bs = 64, 4
    rows = [[] for _ in range(nbr * bs)]
    for br in range(nbr):
        bcs = np.sort(rng.choice(nbr, 6, replace=False))
        for b in bcs:
            mask = rng.random((bs, bs)) < rng.uniform(0.3, 1.0)
            mask[rng.integers(bs), rng.integers(bs)] = True
            for i in range(bs):
                for j in range(bs):
                    if mask[i, j]:
                        rows[br * bs + i].append(b * bs + j)
    mats["randbsr64"] = from_rows(nbr * bs, nbr * bs, rows)

    # ragged edge case: rows not a multiple of 4, a dense row, wide columns
    n = 203
    cols = 33001  # wider than the reference's 32,768-column bitmask window
    rr = []
    for i in range(n):
        if i == 17:
            rr.append(np.sort(rng.choice(cols, 900, replace=False)))
        elif i % 11 == 0:
            rr.append([])
        else:
            rr.append(np.sort(rng.choice(cols, int(rng.integers(1, 12)), replace=False)))
    mats["ragged203"] = from_rows(n, cols, rr)
    return mats


def run_spmv(name, m) -> None:
    lib = C.CDLL(str(pyoracle.REF_DIR / "libref_host.so"))
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, m["cols"])
    rp64 = m["rowptr"].astype(np.int64)
    ci64 = m["colidx"].astype(np.int64)
    y64 = np.zeros(m["rows"])
    lib.ref_spmv_fp64_c.argtypes = [C.c_void_p] * 5 + [C.c_int64, C.c_int64]
    lib.ref_spmv_fp64_c(_p(rp64), _p(ci64), _p(m["values"]), _p(x), _p(y64), m["rows"], m["cols"])
    v32 = m["values"].astype(np.float32)
    x32 = x.astype(np.float32)
    y32 = np.zeros(m["rows"], np.float32)
    lib.ref_spmv_fp32_c.argtypes = [C.c_void_p] * 5 + [C.c_int32, C.c_int32]
    lib.ref_spmv_fp32_c(_p(m["rowptr"]), _p(m["colidx"]), _p(v32), _p(x32), _p(y32), m["rows"], m["cols"])
    y16 = np.zeros(m["rows"], np.float32)
    lib.ref_spmv_fp16_c.argtypes = [C.c_void_p] * 5 + [C.c_int32, C.c_int32]
    lib.ref_spmv_fp16_c(_p(m["rowptr"]), _p(m["colidx"]), _p(v32), _p(x32), _p(y16), m["rows"], m["cols"])
    np.savez_compressed(OUT / f"spmv_{name}.npz", rows=m["rows"], cols=m["cols"], rowptr=m["rowptr"],
                        colidx=m["colidx"], values=m["values"], x=x, y_fp64=y64, y_fp32=y32, y_fp16=y16)


class RefBcsr(C.Structure):
    _fields_ = [("rowRegions", C.c_int32), ("colRegions", C.c_int32), ("nonzeroBlocks", C.c_int32),
                ("blockNum", C.c_int32), ("rowPtr", C.POINTER(C.c_int32)), ("colIdx", C.POINTER(C.c_int32)),
                ("mapping", C.POINTER(C.c_int32)), ("values", C.POINTER(C.c_double))]


class RefDbsr(C.Structure):
    _fields_ = [("row", C.c_int32), ("col", C.c_int32), ("nnz", C.c_int32), ("blc_row", C.c_int32),
                ("blocknnz", C.c_int32), ("warpnum", C.c_int32), ("blcPtr", C.POINTER(C.c_int32)),
                ("colIdx", C.POINTER(C.c_int32)), ("blcVal", C.POINTER(C.c_double)),
                ("blcMap", C.POINTER(C.c_uint16)), ("recorderMap", C.POINTER(C.c_int32)),
                ("prefix", C.POINTER(C.c_int32))]


def _arr(ptr, n, dt):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).copy() if n > 0 else np.zeros(0, dt)


def run_bcsr(name, m, tm, tk) -> None:
    lib = C.CDLL(str(pyoracle.REF_DIR / "libref_host.so"))
    lib.ref_csr2bcsr_c.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_int32, C.POINTER(RefBcsr)]
    o = RefBcsr()
    lib.ref_csr2bcsr_c(m["rows"], m["cols"], m["colidx"].size, _p(m["rowptr"]), _p(m["colidx"]),
                       _p(m["values"]), tm, tk, C.byref(o))
    nb = o.nonzeroBlocks
    np.savez_compressed(OUT / f"bcsr_{name}_{tm}x{tk}.npz", rows=m["rows"], cols=m["cols"], rowptr=m["rowptr"],
                        colidx=m["colidx"], values=m["values"], tile_m=tm, tile_k=tk, rowRegions=o.rowRegions,
                        colRegions=o.colRegions, nonzeroBlocks=nb,
                        bcsrRowPtr=_arr(o.rowPtr, o.rowRegions + 1, np.int32),
                        bcsrColIdx=_arr(o.colIdx, nb, np.int32),
                        mapping=_arr(o.mapping, o.rowRegions * o.colRegions, np.int32),
                        bcsrVal=_arr(o.values, nb * tm * tk, np.float64))


def balance_in_bounds(blcPtr: np.ndarray, cap: int = 64) -> bool:
    """True when balanceDbsr's second walk (include/dbsr.h:139-155) stays
    inside the warp vector its first walk (:103-128) sized.  Outside that the
    reference indexes past the vector (undefined behaviour), so it is not
    run there."""
    lens = np.diff(blcPtr)
    now = 0
    wc = 0
    for L in lens:
        if now + L <= cap:
            now += L
        else:
            if now:
                wc += 1
                now = 0
            if L <= cap:
                now = L
            else:
                wc += (L + cap - 1) // cap
    if now:
        wc += 1
    nw = 0
    for L in lens:
        if now + L <= cap:
            now += L
        else:
            now = 0
            nw += 1 if L <= cap else (L + cap - 1) // cap
        if nw >= wc:
            return False
    return True


def run_dbsr(name, m) -> None:
    lib = C.CDLL(str(pyoracle.REF_DIR / "libref_host.so"))
    P = C.POINTER
    lib.ref_recorder_self_c.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                        P(P(C.c_int32)), P(P(C.c_int32)), P(P(C.c_double))]
    lib.ref_csr2dbsr_c.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   P(RefDbsr)]
    lib.ref_balance_dbsr_c.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, P(C.c_int32),
                                       P(P(C.c_int32))]
    lib.ref_csr2dbsr_recorder_c.argtypes = lib.ref_csr2dbsr_c.argtypes
    rows, cols, nnz = m["rows"], m["cols"], m["colidx"].size
    rrp, rci, rva = P(C.c_int32)(), P(C.c_int32)(), P(C.c_double)()
    lib.ref_recorder_self_c(rows, cols, nnz, _p(m["rowptr"]), _p(m["colidx"]), _p(m["values"]), C.byref(rrp),
                            C.byref(rci), C.byref(rva))
    rec = dict(rowptr=_arr(rrp, rows + 1, np.int32), colidx=_arr(rci, nnz, np.int32), values=_arr(rva, nnz, np.float64))
    for tag, csr in (("plain", m), ("rec", rec)):
        o = RefDbsr()
        lib.ref_csr2dbsr_c(rows, cols, nnz, _p(csr["rowptr"]), _p(csr["colidx"]), _p(csr["values"]), C.byref(o))
        nblk = o.blocknnz // 16
        blcPtr = _arr(o.blcPtr, o.blc_row + 1, np.int32)
        extra = {}
        ok = balance_in_bounds(blcPtr)
        if ok:
            wn = C.c_int32()
            pre = P(C.c_int32)()
            lib.ref_balance_dbsr_c(rows, cols, nnz, o.blc_row, _p(blcPtr), C.byref(wn), C.byref(pre))
            extra["warpnum"] = wn.value
            extra["prefix"] = _arr(pre, wn.value + 1, np.int32)
            if tag == "rec":
                o2 = RefDbsr()
                lib.ref_csr2dbsr_recorder_c(rows, cols, nnz, _p(m["rowptr"]), _p(m["colidx"]), _p(m["values"]),
                                            C.byref(o2))
                extra["recorderMap"] = _arr(o2.recorderMap, rows, np.int32)
        if tag == "rec":
            extra.update(rec_rowptr=rec["rowptr"], rec_colidx=rec["colidx"], rec_values=rec["values"])
        np.savez_compressed(OUT / f"dbsr_{name}_{tag}.npz", rows=rows, cols=cols, rowptr=m["rowptr"],
                            colidx=m["colidx"], values=m["values"], blc_row=o.blc_row, blocknnz=o.blocknnz,
                            balance_in_bounds=int(ok), blcPtr=blcPtr, colIdx_d=_arr(o.colIdx, o.blocknnz, np.int32),
                            blcVal=_arr(o.blcVal, o.blocknnz, np.float64), blcMap=_arr(o.blcMap, nblk, np.uint16),
                            **extra)


def run_dasp(name, m, threshold=0.75, block_longest=256) -> None:
    x = np.random.default_rng(11).uniform(-1, 1, m["cols"])
    rec = pyoracle.run_capture("dasp_capture", m["rows"], m["cols"], m["rowptr"], m["colidx"], m["values"], x,
                               threshold, block_longest)
    out = dict(rows=m["rows"], cols=m["cols"], rowptr=m["rowptr"], colidx=m["colidx"], values=m["values"], x=x,
               threshold=threshold, block_longest=block_longest)
    ints = {"long_ptr_warp", "reg_cid", "block_ptr", "irreg_cid", "irreg_rpt", "short_cid", "long_cid", "order_rid"}
    for k, v in rec.items():
        kind, nm = k.split(":", 1)
        if kind == "int":
            out["int_" + nm] = np.frombuffer(v, np.int32)[0]
        elif nm in ints:
            out["arr_" + nm] = np.frombuffer(v, np.int32).copy()
        elif nm in ("dX_val", "dY_val", "warp_val"):
            continue  # x, zeros and kernel scratch
        else:
            out["arr_" + nm] = np.frombuffer(v, np.float64).copy()
    np.savez_compressed(OUT / f"dasp_{name}_t{int(threshold * 100)}_l{block_longest}.npz", **out)


def run_amgt(name, m) -> None:
    x = np.zeros(m["cols"])
    rec = pyoracle.run_capture("amgt_capture", m["rows"], m["cols"], m["rowptr"], m["colidx"], m["values"], x)
    ints = np.frombuffer(rec["ints:row,col,nnz,blc_row,blc_col,blc_num"], np.int32)
    np.savez_compressed(OUT / f"amgt_{name}.npz", rows=m["rows"], cols=m["cols"], rowptr=m["rowptr"],
                        colidx=m["colidx"], values=m["values"], blc_row=ints[3], blc_col=ints[4], blc_num=ints[5],
                        nnz_field=ints[2], stand=np.frombuffer(rec["f64:stand"], np.float64)[0],
                        avg_nnz=np.frombuffer(rec["f64:avg_nnz"], np.float64)[0],
                        warpnum=np.frombuffer(rec["int:warpnum"], np.int32)[0],
                        blcPtr=np.frombuffer(rec["arr:blcPtr"], np.int32),
                        blcIdx=np.frombuffer(rec["arr:blcIdx"], np.int32),
                        blcVal=np.frombuffer(rec["arr:blcVal"], np.float64),
                        blcMap=np.frombuffer(rec["arr:blcMap"], np.uint16),
                        rowPtrbyWarp=np.frombuffer(rec["arr:rowPtrbyWarp"], np.int32),
                        rowIdxbyWarp=np.frombuffer(rec["arr:rowIdxbyWarp"], np.int32))


def run_blockinfo() -> None:
    """bench/blockinfo.cpp (oracle/_ref/blockinfo) on matrices regenerated
    from the library's seeded generators (names match tests/test_oracle.py)."""
    import benchsp_b200 as bsp
    mats = {"powerlaw": bsp.gen_powerlaw(30000, 2.0, 10000, 17), "laplace": bsp.gen_laplace2d(64, 80),
            "random": bsp.gen_random_bsr(1000, 4, 8, 0.3, 1.0, 5)}
    names, b, br = [], [], []
    for name, A in mats.items():
        r = pyoracle.run_ref_blockinfo(A.rows, A.cols, A.rowptr, A.colidx, A.values)
        names.append(name)
        b.append(r["blocks"])
        br.append(r["blocks_recorder"])
    np.savez_compressed(OUT / "blockinfo_ref.npz", names=np.array(names), blocks=np.array(b),
                        blocks_recorder=np.array(br))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--amgt", action="store_true", help="only the AmgT fixtures (needs a GPU)")
    a = ap.parse_args()
    mats = matrices()
    if a.amgt:
        for name, m in mats.items():
            run_amgt(name, m)
        return
    if not pyoracle.ref_available():
        raise SystemExit("oracle/_ref is not built (needs the reference sources): make -C oracle")
    for name, m in mats.items():
        run_spmv(name, m)
        run_dasp(name, m)
        run_dbsr(name, m)
    run_dasp("powerlaw2k", mats["powerlaw2k"], 0.5, 64)
    for name in ("lap16", "randbsr64", "powerlaw2k"):
        run_bcsr(name, mats[name], 4, 4)
    run_bcsr("randbsr64", mats["randbsr64"], 16, 16)
    run_bcsr("lap16", mats["lap16"], 3, 3)
    run_blockinfo()


if __name__ == "__main__":
    main()
