"""The reference's own SpMV kernels, compiled for sm_100a from src/amgT.cu and
src/csrspmv.cu (oracle/_ref/ref_amgt_time, ref_csr_time) and called
directly on the B200: their results agree with the oracle's FP64 SpMV within
the rounding bound, as do the library's, and the two are timed on the same
arrays (printed as one JSON line per case; run with -s to see them).

The AmgT kernels get the BSR arrays built by the library's converter, which
are bit-identical to the reference's CSR2BSR_GPU (test_bsr_gpu.py pins that),
so the reference's hash-based conversion is not run at these sizes."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _exe(name):
    p = pyoracle.REF_DIR / name
    if not p.exists():
        pytest.skip(f"{name} not built (needs the reference sources at build time)")
    return str(p)


def _events(fn, reps, flush=None):
    import torch
    for _ in range(5):
        fn()
    torch.cuda.synchronize()
    if flush is None:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) * 1e3 / reps
    t = []
    for i in range(reps):
        flush.fill_(i & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        t.append(a.elapsed_time(b) * 1e3)
    return float(np.median(t))


def amgt_case(cuda, grid, reps=50):
    """Runs the reference's four AmgT BSR kernels and the library's FFMA BSR
    kernel on the 27-point stencil (grid^3 nodes x 4 dof); returns the record
    and the results."""
    import torch
    A = bsp.gen_stencil27(grid, 4, 20261204)
    x = bsp.gen_uniform(A.cols, 7)
    rp, ci, va, xd = (torch.from_numpy(a).to(cuda) for a in (A.rowptr, A.colidx, A.values, x))
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    arr = M.arrays()
    names = ["bsr_spmv_tc_fp64", "bsr_spmv_cc_fp64", "bsr_spmv_balanced_tc_fp64", "bsr_spmv_balanced_cc_fp64"]
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([A.rows, A.cols, M.blc_row, M.blc_col, M.blc_num, M.warpnum], np.int32).tofile(f)
            for k in ("blcPtr", "blcIdx", "blcVal", "blcMap", "rowPtrbyWarp", "rowIdxbyWarp"):
                arr[k].tofile(f)
            x.tofile(f)
        del arr
        r = subprocess.run([_exe("ref_amgt_time"), fin, fout, str(reps)], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr
        times = json.loads(r.stdout.strip().splitlines()[-1])
        ys = np.fromfile(fout, np.float64).reshape(len(names), A.rows)
    y = torch.empty(A.rows, dtype=torch.float64, device=cuda)
    ours = _events(lambda: M.spmv(xd, y), reps)
    M.spmv(xd, y)
    torch.cuda.synchronize()
    rec = {"case": f"amgt_stencil27_{grid}cubed_4dof", "n": A.rows, "nnz": A.nnz, "blocks": M.blc_num,
           "reference_us": times, "ours_us": round(ours, 2),
           "speedup_vs_reference_tc": round(times["bsr_spmv_tc_fp64"] / ours, 2)}
    M.free()
    return rec, A, x, dict(zip(names, ys)), y.cpu().numpy()


@pytest.mark.parametrize("grid", [40])
def test_reference_amgt_kernels_agree_and_are_timed(cuda, grid):
    rec, A, x, ys, ours = amgt_case(cuda, grid)
    want = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    for name, yr in ys.items():
        assert np.all(np.abs(yr - want) <= tol), name
    assert np.all(np.abs(ours - want) <= tol)
    print(json.dumps(rec))


def csr_case(cuda, A, reps=50, flush_mb=256):
    """Runs the reference's spmv_fp64 (thread per row) and spmv_fp64_balance
    kernels and the library's CSR SpMV on A, L2 flushed between launches."""
    import torch
    x = bsp.gen_uniform(A.cols, 9)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([A.rows, A.cols, A.nnz], np.int32).tofile(f)
            for a in (A.rowptr, A.colidx, A.values, x):
                a.tofile(f)
        r = subprocess.run([_exe("ref_csr_time"), fin, fout, str(reps), str(flush_mb)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        times = json.loads(r.stdout.strip().splitlines()[-1])
        ys = np.fromfile(fout, np.float64).reshape(2, A.rows)
    rp, ci, va, xd = (torch.from_numpy(a).to(cuda) for a in (A.rowptr, A.colidx, A.values, x))
    y = torch.empty(A.rows, dtype=torch.float64, device=cuda)
    flush = torch.empty(flush_mb << 20, dtype=torch.uint8, device=cuda)
    ours = _events(lambda: bsp.csr_spmv(rp, ci, va, xd, y), reps, flush)
    bsp.csr_spmv(rp, ci, va, xd, y)
    torch.cuda.synchronize()
    rec = {"reference_us": times, "ours_us": round(ours, 2),
           "speedup_vs_reference_spmv_fp64": round(times["spmv_fp64"] / ours, 2)}
    return rec, x, {"spmv_fp64": ys[0], "spmv_fp64_balance": ys[1]}, y.cpu().numpy()


def test_reference_csr_kernels_agree_and_are_timed(cuda):
    A = bsp.gen_laplace2d(512, 512)
    rec, x, ys, ours = csr_case(cuda, A)
    want = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    assert np.all(np.abs(ys["spmv_fp64"] - want) <= tol)
    assert np.all(np.abs(ys["spmv_fp64_balance"] - want) <= tol)
    assert np.all(np.abs(ours - want) <= tol)
    rec["case"] = "csr_laplace2d_512_l2_flushed"
    rec["n"], rec["nnz"] = A.rows, A.nnz
    print(json.dumps(rec))


def dasp_case(cuda, A, reps=50):
    """Runs the reference's DASP kernels (dasp_spmv2<1> + longPart_sum) on the
    arguments its spmv_all builds for A (captured by oracle/_ref/dasp_capture)
    and the library's DASP SpMV on its own packing (bit-identical to those
    arrays); returns the record, x, the reference's y (original row order)
    and the library's y."""
    import torch
    x = bsp.gen_uniform(A.cols, 13)
    with tempfile.TemporaryDirectory() as td:
        fin, fcap, fout = (os.path.join(td, n) for n in ("in.bin", "cap.bin", "y.bin"))
        pyoracle.write_csr_bin(fin, A.rows, A.cols, A.rowptr, A.colidx, A.values, x)
        r = subprocess.run([_exe("dasp_capture"), fin, fcap], capture_output=True, text=True, timeout=1200)
        assert r.returncode == 0, r.stderr
        order = np.frombuffer(pyoracle.read_records(fcap)["arr:order_rid"], np.int32)
        r = subprocess.run([_exe("ref_dasp_time"), fcap, fout, str(reps)], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr
        times = json.loads(r.stdout.strip().splitlines()[-1])
        y_perm = np.fromfile(fout, np.float64)[:A.rows]
    y_ref = np.empty(A.rows)
    y_ref[order] = y_perm                          # output position k holds row order_rid[k]
    rp, ci, va, xd = (torch.from_numpy(a).to(cuda) for a in (A.rowptr, A.colidx, A.values, x))
    D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols)
    y = torch.empty(A.rows, dtype=torch.float64, device=cuda)
    # the reference writes y in order_rid order: time that form too
    ours_perm = _events(lambda: D.spmv(xd, y, permuted=True), reps)
    ours = _events(lambda: D.spmv(xd, y), reps)
    D.spmv(xd, y)
    torch.cuda.synchronize()
    rec = {"reference_us": times, "ours_us_permuted_output": round(ours_perm, 2),
           "ours_us_row_order": round(ours, 2),
           "speedup_same_output_order": round(times["dasp_spmv2+longPart_sum"] / ours_perm, 2)}
    D.free()
    return rec, x, y_ref, y.cpu().numpy()


def test_reference_dasp_kernels_agree_and_are_timed(cuda):
    A = bsp.gen_powerlaw(1 << 17, 2.0, 4000, 21)
    rec, x, y_ref, ours = dasp_case(cuda, A)
    want = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    assert np.all(np.abs(y_ref - want) <= tol)
    assert np.all(np.abs(ours - want) <= tol)
    rec["case"] = "dasp_powerlaw_2^17_zipf2"
    rec["n"], rec["nnz"] = A.rows, A.nnz
    print(json.dumps(rec))
