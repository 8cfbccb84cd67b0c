"""Device CSR->BSR conversion (bit-exact with the reference's CSR2BSR_GPU
ordering) and BSR SpMV against the oracle."""
import glob
from pathlib import Path

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
SPMV = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "spmv_*.npz")))


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _check_arrays(M, o):
    a = M.arrays()
    for k in ("blcPtr", "blcIdx", "blcVal", "rowPtrbyWarp", "rowIdxbyWarp"):
        assert np.array_equal(a[k], o[k]), k
    assert np.array_equal(a["blcMap"].astype(np.uint64), o["blcMap"].astype(np.uint64))
    assert M.blc_num == o["blc_num"] and M.warpnum == o["warpnum"]
    assert abs(M.stand - o["stand"]) <= 1e-6 * max(1.0, o["stand"])
    assert M.avg_nnz == pytest.approx(o["avg_nnz"], rel=1e-15)


@pytest.mark.parametrize("name", SPMV)
@pytest.mark.parametrize("bs", [4, 8])
def test_csr2bsr_bit_exact(cuda, golden, name, bs):
    g = golden(name)
    rows, cols = int(g["rows"]), int(g["cols"])
    rp, ci, va = _dev(cuda, g["rowptr"], g["colidx"], g["values"])
    M = bsp.csr2bsr(rp, ci, va, rows=rows, cols=cols, bs=bs)
    _check_arrays(M, pyoracle.csr2bsr(rows, cols, g["rowptr"], g["colidx"], g["values"], bs))
    assert M.nnz == M.blc_num * bs * bs and M.blc_row == -(-rows // bs)


def test_csr2bsr_matches_reference_gpu_conversion(cuda):
    """Runs the reference's own CSR2BSR_GPU (oracle/_ref/amgt_capture) on the
    same inputs when it has been built."""
    exe = pyoracle.REF_DIR / "amgt_capture"
    if not exe.exists():
        pytest.skip("oracle/_ref/amgt_capture not built")
    for name in SPMV:
        g = dict(np.load(GOLDEN / name))
        rows, cols = int(g["rows"]), int(g["cols"])
        rec = pyoracle.run_capture("amgt_capture", rows, cols, g["rowptr"], g["colidx"], g["values"],
                                   np.zeros(cols))
        rp, ci, va = _dev(cuda, g["rowptr"], g["colidx"], g["values"])
        a = bsp.csr2bsr(rp, ci, va, rows=rows, cols=cols, bs=4).arrays()
        for k, dt in (("blcPtr", np.int32), ("blcIdx", np.int32), ("blcVal", np.float64), ("blcMap", np.uint16),
                      ("rowPtrbyWarp", np.int32), ("rowIdxbyWarp", np.int32)):
            assert np.array_equal(a[k], np.frombuffer(rec["arr:" + k], dt)), (name, k)


@pytest.mark.parametrize("kind", ["stencil27", "random4", "random8", "powerlaw"])
def test_csr2bsr_bit_exact_generated(cuda, kind):
    if kind == "stencil27":
        A, bs = bsp.gen_stencil27(12, 4, 1), 4
    elif kind == "random4":
        A, bs = bsp.gen_random_bsr(3000, 4, 16, 0.3, 1.0, 2), 4
    elif kind == "random8":
        A, bs = bsp.gen_random_bsr(1500, 8, 16, 0.3, 1.0, 2), 8
    else:
        A, bs = bsp.gen_powerlaw(40000, 2.0, 10000, 3), 4
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
    _check_arrays(M, pyoracle.csr2bsr(A.rows, A.cols, A.rowptr, A.colidx, A.values, bs))


@pytest.mark.parametrize("kind,bs", [("stencil27", 4), ("stencil27", 8), ("random", 4), ("random", 8),
                                     ("powerlaw", 4), ("ragged", 4)])
@pytest.mark.parametrize("algo", ["ffma", "dmma", "adaptive"])
def test_bsr_spmv_against_oracle(cuda, golden, kind, bs, algo):
    if algo == "dmma" and bs != 4:
        pytest.skip("DMMA path is 4x4")
    if kind == "stencil27":
        A = bsp.gen_stencil27(12, 4, 1)
    elif kind == "random":
        A = bsp.gen_random_bsr(2000, bs, 16, 0.3, 1.0, 2)
    elif kind == "powerlaw":
        A = bsp.gen_powerlaw(30000, 2.0, 3000, 3)
    else:
        g = golden("spmv_ragged203.npz")
        A = bsp.HostCSR(int(g["rows"]), int(g["cols"]), g["rowptr"], g["colidx"], g["values"])
    x = bsp.gen_uniform(A.cols, 77)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
    y = M.spmv(xx, algo=algo).cpu().numpy()
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    err = np.abs(y - ref)
    assert np.all(err <= tol), float(np.max(err - tol))


def test_bsr_spmv_alpha_beta(cuda):
    import torch
    A = bsp.gen_stencil27(8, 4, 5)
    x = bsp.gen_uniform(A.cols, 1)
    y0 = bsp.gen_uniform(A.rows, 2)
    ref = -1.5 * pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x) + 2.0 * y0
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    for algo in ("ffma", "dmma"):
        y = torch.from_numpy(y0.copy()).to(cuda)
        M.spmv(xx, y, alpha=-1.5, beta=2.0, algo=algo)
        tol = 1.5 * pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x) + 8 * 2.0 ** -53 * (np.abs(ref) + 2)
        assert np.all(np.abs(y.cpu().numpy() - ref) <= tol)


def test_misaligned_x_uses_scalar_gathers(cuda):
    import torch
    A = bsp.gen_stencil27(6, 4, 5)
    x = bsp.gen_uniform(A.cols + 1, 1)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x[1:].copy())
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    xx = torch.from_numpy(x).to(cuda)[1:]  # 8-byte aligned only
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    y = M.spmv(xx, algo="ffma").cpu().numpy()
    assert np.all(np.abs(y - ref) <= pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x[1:].copy()))


@pytest.mark.parametrize("kind", ["stencil", "random", "ragged"])
@pytest.mark.parametrize("chunks", [1, 3, 8, 64])
def test_bsr_host_pipelined_matches_host_call(cuda, kind, chunks):
    """The overlapped host-buffer SpMV returns exactly what the plain
    host-buffer call returns (same kernel per row), with and without beta."""
    import torch
    A = {"stencil": lambda: bsp.gen_stencil27(10, 4, 2), "random": lambda: bsp.gen_random_bsr(300, 4, 5, 0.4, 1.0, 3),
         "ragged": lambda: bsp.gen_powerlaw(1001, 1.9, 200, 4)}[kind]()
    rp, ci, va = (torch.from_numpy(a).to(cuda) for a in (A.rowptr, A.colidx, A.values))
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    x = torch.from_numpy(bsp.gen_uniform(A.cols, 5)).pin_memory().numpy()
    y0 = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, A.rows)).pin_memory().numpy()
    want = y0.copy()
    M.spmv_host(x, want, alpha=1.5, beta=-0.5)
    P = M.host_plan(chunks)
    for _ in range(2):
        got = y0.copy()
        P.spmv(x, got, alpha=1.5, beta=-0.5)
        assert np.array_equal(got, want)
    got = np.empty(A.rows)
    P.spmv(x, got)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    assert np.all(np.abs(got - ref) <= pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x))
    # the grid cap of the ranges changes the schedule, not the sums
    for ctas in (0, 1, 37):
        P.set_ctas(ctas)
        got2 = np.empty(A.rows)
        P.spmv(x, got2)
        assert np.array_equal(got2, got), ctas
    with pytest.raises(bsp.BspError):
        P.set_ctas(-1)
    P.close()
    M.free()
