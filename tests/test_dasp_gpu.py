"""Device DASP packing against the arrays the reference's own spmv_all
uploads (captured through oracle/_ref/dasp_capture, committed fixtures and
live runs), and the fused DASP SpMV against the oracle."""
import glob
from pathlib import Path

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
DASP = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "dasp_*.npz")))
ARRS = ("long_val", "long_cid", "long_ptr_warp", "reg_val", "reg_cid", "block_ptr", "irreg_val", "irreg_cid",
        "irreg_rpt", "short_val", "short_cid", "order_rid")
INTS = ("row_long", "row_block", "blocknum", "short_row_1", "common_13", "short_row_34", "short_row_2",
        "offset_reg", "offset_short1", "offset_short13", "offset_short34", "offset_short22",
        "fill0_nnz_short13", "fill0_nnz_short34")


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _check(D, ref: dict):
    a = D.arrays()
    for k in ARRS:
        if ("arr_" + k) in ref:
            assert np.array_equal(a[k], ref["arr_" + k]), k
        else:  # empty in the reference
            assert a[k].size == 0, k
    for k in INTS:
        assert getattr(D, k) == int(ref["int_" + k]), k
    assert D.block_num_all == int(ref["int_grid_all"])


@pytest.mark.parametrize("name", DASP)
def test_dasp_packing_bit_exact_with_reference_fixture(cuda, golden, name):
    g = golden(name)
    rows, cols = int(g["rows"]), int(g["cols"])
    rp, ci, va = _dev(cuda, g["rowptr"], g["colidx"], g["values"])
    D = bsp.csr2dasp(rp, ci, va, rows=rows, cols=cols, threshold=float(g["threshold"]),
                     block_longest=int(g["block_longest"]))
    _check(D, g)


def _capture(rows, cols, rp, ci, va, th, bl):
    rec = pyoracle.run_capture("dasp_capture", rows, cols, rp, ci, va, np.zeros(cols), th, bl)
    out = {}
    ints = {"long_ptr_warp", "reg_cid", "block_ptr", "irreg_cid", "irreg_rpt", "short_cid", "long_cid", "order_rid"}
    for k, v in rec.items():
        kind, nm = k.split(":", 1)
        if kind == "int":
            out["int_" + nm] = np.frombuffer(v, np.int32)[0]
        elif nm in ints:
            out["arr_" + nm] = np.frombuffer(v, np.int32)
        elif nm not in ("dX_val", "dY_val", "warp_val"):
            out["arr_" + nm] = np.frombuffer(v, np.float64)
    return out


@pytest.mark.parametrize("n,alpha,cap,th,bl", [(100000, 2.0, 10000, 0.75, 256), (50000, 1.6, 3000, 0.5, 64),
                                               (30000, 2.5, 600, 0.9, 128)])
def test_dasp_packing_matches_live_reference(cuda, n, alpha, cap, th, bl):
    if not (pyoracle.REF_DIR / "dasp_capture").exists():
        pytest.skip("oracle/_ref/dasp_capture not built")
    A = bsp.gen_powerlaw(n, alpha, cap, 31)
    ref = _capture(A.rows, A.cols, A.rowptr, A.colidx, A.values, th, bl)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols, threshold=th, block_longest=bl)
    _check(D, ref)


@pytest.mark.parametrize("kind", ["powerlaw", "powerlaw_heavy", "laplace", "ragged", "lap16"])
def test_dasp_spmv(cuda, golden, kind):
    import torch
    if kind in ("ragged", "lap16"):
        g = golden(f"spmv_{'ragged203' if kind == 'ragged' else 'lap16'}.npz")
        A = bsp.HostCSR(int(g["rows"]), int(g["cols"]), g["rowptr"], g["colidx"], g["values"])
    else:
        A = {"powerlaw": lambda: bsp.gen_powerlaw(200000, 2.0, 10000, 5),
             "powerlaw_heavy": lambda: bsp.gen_powerlaw(100000, 1.5, 50000, 6),
             "laplace": lambda: bsp.gen_laplace2d(200, 300)}[kind]()
    x = bsp.gen_uniform(A.cols, 8)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols)
    chunks = np.diff(D.arrays()["long_ptr_warp"])
    assert D.long_groups == int(np.sum((chunks + 3) // 4))   # up to 4 chunks of a row per warp
    for _ in range(3):  # repeated calls reuse the long-row counters
        y = D.spmv(xx).cpu().numpy()
        assert np.all(np.abs(y - ref) <= tol)
    yp = D.spmv(xx, permuted=True).cpu().numpy()
    order = D.arrays()["order_rid"]
    assert np.all(np.abs(yp - ref[order]) <= tol[order])
    y0 = torch.ones(A.rows, dtype=torch.float64, device=cuda)
    yb = D.spmv(xx, y0, alpha=-2.0, beta=0.5).cpu().numpy()
    refb = -2.0 * ref + 0.5
    assert np.all(np.abs(yb - refb) <= 2 * tol + 4 * 2.0 ** -53 * (np.abs(refb) + 1))


def test_dasp_rejects_zero_threshold(cuda):
    A = bsp.gen_laplace2d(8, 8)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    with pytest.raises(bsp.BspError):
        bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols, threshold=0.0)
