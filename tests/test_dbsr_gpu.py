"""Device DBSR conversion (bit-exact with include/dbsr.h's converters) and
DBSR SpMV (A*x, not the reference kernels' row sums) against the oracle."""
import glob
from pathlib import Path

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
DBSR = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "dbsr_*.npz")))


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _compare(M, o, rec):
    a = M.arrays()
    assert M.blc_row == o["blc_row"] and M.blocknnz == o["blocknnz"]
    for k in ("blcPtr", "colIdx", "blcVal", "blcMap", "prefix"):
        assert np.array_equal(a[k], o[k]), k
    assert M.warpnum == o["warpnum"] and M.balance_overflow == o["balance_overflow"]
    if rec:
        assert np.array_equal(a["recorderMap"], o["recorderMap"])


@pytest.mark.parametrize("name", DBSR)
def test_csr2dbsr_bit_exact_with_reference_fixture(cuda, golden, name):
    g = golden(name)
    rec = name.endswith("_rec.npz")
    rows, cols = int(g["rows"]), int(g["cols"])
    rp, ci, va = _dev(cuda, g["rowptr"], g["colidx"], g["values"])
    M = bsp.csr2dbsr(rp, ci, va, rows=rows, cols=cols, recorder=rec)
    a = M.arrays()
    assert np.array_equal(a["blcPtr"], g["blcPtr"])
    assert np.array_equal(a["colIdx"], g["colIdx_d"])
    assert np.array_equal(a["blcVal"], g["blcVal"])
    assert np.array_equal(a["blcMap"], g["blcMap"])
    if int(g["balance_in_bounds"]):
        assert M.warpnum == int(g["warpnum"]) and M.balance_overflow == 0
        assert np.array_equal(a["prefix"], g["prefix"])
        if rec:
            assert np.array_equal(a["recorderMap"], g["recorderMap"])
    else:
        assert M.balance_overflow == 1
    _compare(M, pyoracle.csr2dbsr(g["rowptr"], g["colidx"], g["values"], rec), rec)


@pytest.mark.parametrize("kind", ["powerlaw", "laplace", "random"])
@pytest.mark.parametrize("rec", [True, False])
def test_csr2dbsr_generated(cuda, kind, rec):
    A = {"powerlaw": lambda: bsp.gen_powerlaw(60000, 2.0, 10000, 4),
         "laplace": lambda: bsp.gen_laplace2d(300, 301),
         "random": lambda: bsp.gen_random_bsr(4000, 4, 16, 0.3, 1.0, 8)}[kind]()
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    M = bsp.csr2dbsr(rp, ci, va, rows=A.rows, cols=A.cols, recorder=rec)
    _compare(M, pyoracle.csr2dbsr(A.rowptr, A.colidx, A.values, rec), rec)


@pytest.mark.parametrize("kind", ["powerlaw", "laplace", "random", "ragged"])
@pytest.mark.parametrize("rec", [True, False])
def test_dbsr_spmv(cuda, golden, kind, rec):
    import torch
    if kind == "ragged":
        g = golden("spmv_ragged203.npz")
        A = bsp.HostCSR(int(g["rows"]), int(g["cols"]), g["rowptr"], g["colidx"], g["values"])
    else:
        A = {"powerlaw": lambda: bsp.gen_powerlaw(60000, 2.0, 10000, 4),
             "laplace": lambda: bsp.gen_laplace2d(300, 301),
             "random": lambda: bsp.gen_random_bsr(4000, 4, 16, 0.3, 1.0, 8)}[kind]()
    x = bsp.gen_uniform(A.cols, 3)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2dbsr(rp, ci, va, rows=A.rows, cols=A.cols, recorder=rec)
    y = M.spmv(xx).cpu().numpy()
    assert np.all(np.abs(y - ref) <= tol)
    if rec:
        yp = M.spmv(xx, permuted=True).cpu().numpy()
        order = M.arrays()["recorderMap"]
        assert np.all(np.abs(yp - ref[order]) <= tol[order])
    y0 = torch.from_numpy(x[:A.rows].copy() if A.cols >= A.rows else np.ones(A.rows)).to(cuda)
    yb = M.spmv(xx, y0.clone(), alpha=2.0, beta=-1.0).cpu().numpy()
    refb = 2.0 * ref - y0.cpu().numpy()
    assert np.all(np.abs(yb - refb) <= 2 * tol + 4 * 2.0 ** -53 * (np.abs(refb) + 1))
