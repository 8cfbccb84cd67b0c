"""CSR SpMV kernels on the GPU against the oracle (src/ref.cpp restated) and
the reference's own outputs in tests/golden."""
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


def _within(y, ref, tol):
    err = np.abs(y - ref)
    assert np.all(err <= tol), f"max excess {np.max(err - tol)} at {int(np.argmax(err - tol))}"


@pytest.mark.parametrize("name", SPMV)
def test_scalar_fp64_is_bit_exact_with_reference(cuda, golden, name):
    g = golden(name)
    rp, ci, va, x = _dev(cuda, g["rowptr"], g["colidx"], g["values"], g["x"])
    y = bsp.csr_spmv(rp, ci, va, x, algo="scalar").cpu().numpy()
    assert np.array_equal(y.view(np.uint64), g["y_fp64"].view(np.uint64))


@pytest.mark.parametrize("name", SPMV)
def test_stream_is_bit_exact_with_reference(cuda, golden, name):
    """The warp-per-32-rows stream kernel sums each row left to right with
    separately rounded multiply and add: the reference's own results, bit for
    bit, in FP64, FP32 and FP16."""
    import torch
    g = golden(name)
    rp, ci, va, x = _dev(cuda, g["rowptr"], g["colidx"], g["values"], g["x"])
    y = bsp.csr_spmv(rp, ci, va, x, algo="stream").cpu().numpy()
    assert np.array_equal(y.view(np.uint64), g["y_fp64"].view(np.uint64))
    v32 = torch.from_numpy(g["values"].astype(np.float32)).to(cuda)
    x32 = torch.from_numpy(g["x"].astype(np.float32)).to(cuda)
    y32 = bsp.csr_spmv(rp, ci, v32, x32, algo="stream").cpu().numpy()
    assert np.array_equal(y32.view(np.uint32), g["y_fp32"].view(np.uint32))
    y16 = bsp.csr_spmv(rp, ci, v32.half(), x32.half(), algo="stream").float().cpu().numpy()
    assert np.array_equal(y16.view(np.uint32), g["y_fp16"].view(np.uint32))


def test_stream_long_rows_bit_exact(cuda):
    """Rows far longer than a 256-entry piece (and warps whose 32 rows span
    many pieces) give the scalar kernel's results exactly."""
    A = bsp.gen_powerlaw(200000, 1.6, 100000, 12)
    assert np.diff(A.rowptr).max() > 10000
    x = bsp.gen_uniform(A.cols, 13)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    y = bsp.csr_spmv(rp, ci, va, xx, algo="stream").cpu().numpy()
    assert np.array_equal(y, ref)
    ys = bsp.csr_spmv(rp, ci, va, xx, algo="scalar").cpu().numpy()
    assert np.array_equal(y, ys)


@pytest.mark.parametrize("rows", [1, 31, 33, 1000])
def test_stream_ragged_tail_warp(cuda, rows):
    """Row counts that leave the last warp partly empty."""
    rng = np.random.default_rng(rows)
    lens = rng.integers(0, 40, rows)
    rp = np.zeros(rows + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    cols = 500
    ci = np.concatenate([np.sort(rng.choice(cols, l, replace=False)) for l in lens]).astype(np.int32)
    va = rng.standard_normal(ci.size)
    x = rng.uniform(-1, 1, cols)
    ref = pyoracle.spmv_f64(rp, ci, va, x)
    d = _dev(cuda, rp, ci, va, x)
    y = bsp.csr_spmv(*d, algo="stream").cpu().numpy()
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("name", SPMV)
@pytest.mark.parametrize("algo,lanes", [("vector", 0), ("vector", 1), ("vector", 4), ("vector", 32),
                                        ("merge", 0)])
def test_fp64_kernels_within_rounding_bound(cuda, golden, name, algo, lanes):
    g = golden(name)
    rp, ci, va, x = _dev(cuda, g["rowptr"], g["colidx"], g["values"], g["x"])
    y = bsp.csr_spmv(rp, ci, va, x, algo=algo, lanes=lanes).cpu().numpy()
    tol = pyoracle.spmv_tolerance(g["rowptr"], g["colidx"], g["values"], g["x"])
    _within(y, g["y_fp64"], tol)


@pytest.mark.parametrize("name", SPMV)
def test_scalar_fp32_and_fp16_bit_exact_with_reference(cuda, golden, name):
    import torch
    g = golden(name)
    rp, ci = _dev(cuda, g["rowptr"], g["colidx"])
    v32 = torch.from_numpy(g["values"].astype(np.float32)).to(cuda)
    x32 = torch.from_numpy(g["x"].astype(np.float32)).to(cuda)
    y32 = bsp.csr_spmv(rp, ci, v32, x32, algo="scalar").cpu().numpy()
    assert np.array_equal(y32.view(np.uint32), g["y_fp32"].view(np.uint32))
    y16 = bsp.csr_spmv(rp, ci, v32.half(), x32.half(), algo="scalar").float().cpu().numpy()
    assert np.array_equal(y16.view(np.uint32), g["y_fp16"].view(np.uint32))


@pytest.mark.parametrize("dt", ["float32", "float16", "bfloat16"])
def test_reduced_precision_vector_kernels(cuda, dt):
    import torch
    A = bsp.gen_powerlaw(50000, 2.0, 2000, 5)
    x = bsp.gen_uniform(A.cols, 6)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tdt = getattr(torch, dt)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    v = torch.from_numpy(A.values).to(cuda).to(tdt)
    xx = torch.from_numpy(x).to(cuda).to(tdt)
    y = bsp.csr_spmv(rp, ci, v, xx).double().cpu().numpy()
    # storage rounding of values and x (2 * unit) plus FP32 accumulation
    unit = {"float32": 2.0 ** -24, "float16": 2.0 ** -11, "bfloat16": 2.0 ** -8}[dt]
    scale = pyoracle.abs_rowsum(A.rowptr, A.colidx, A.values, x)
    out_round = unit * np.abs(ref)
    tol = (3 * unit + 2 * np.diff(A.rowptr) * 2.0 ** -24) * scale + out_round + 1e-30
    _within(y, ref, tol * 1.01)


@pytest.mark.parametrize("algo", ["vector", "merge", "scalar", "stream"])
def test_laplace_512_config(cuda, algo):
    A = bsp.gen_laplace2d(512, 512)
    x = bsp.gen_uniform(A.cols, 20261203)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    y = bsp.csr_spmv(rp, ci, va, xx, algo=algo).cpu().numpy()
    if algo in ("scalar", "stream"):
        assert np.array_equal(y, ref)
    else:
        _within(y, ref, pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x))


def test_merge_path_power_law_long_rows(cuda):
    A = bsp.gen_powerlaw(200000, 1.6, 100000, 12)
    assert np.diff(A.rowptr).max() > 10000
    x = bsp.gen_uniform(A.cols, 13)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    _within(bsp.csr_spmv_merge(rp, ci, va, xx).cpu().numpy(), ref, tol)
    # lanes 1 / 4 / auto: rows above 64 entries per lane go to the whole warp
    for lanes in (32, 4, 1, 0):
        _within(bsp.csr_spmv(rp, ci, va, xx, algo="vector", lanes=lanes).cpu().numpy(), ref, tol)


@pytest.mark.parametrize("lanes", [1, 2, 8])
def test_vector_warp_rows_alpha_beta(cuda, lanes):
    """Rows just above and below the whole-warp threshold (64 entries per
    lane), with alpha and beta, in every position of a warp's row group."""
    import torch
    rng = np.random.default_rng(lanes)
    n, cols = 700, 5000
    lens = rng.integers(0, 8, n)
    thr = 64 * lanes
    lens[rng.choice(n, 60, replace=False)] = rng.choice([thr - 1, thr, thr + 1, 3 * thr + 7], 60)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(cols, l, replace=False)) for l in lens]).astype(np.int32)
    va = rng.standard_normal(ci.size)
    x = rng.uniform(-1, 1, cols)
    y0 = rng.uniform(-1, 1, n)
    ref = 1.5 * pyoracle.spmv_f64(rp, ci, va, x) + 0.25 * y0
    d = _dev(cuda, rp, ci, va, x)
    y = torch.from_numpy(y0.copy()).to(cuda)
    bsp.csr_spmv(*d, y=y, alpha=1.5, beta=0.25, algo="vector", lanes=lanes)
    tol = 1.5 * pyoracle.spmv_tolerance(rp, ci, va, x) + 4 * 2.0 ** -53 * (np.abs(ref) + 1)
    _within(y.cpu().numpy(), ref, tol)


@pytest.mark.parametrize("algo", ["vector", "merge", "scalar", "stream"])
def test_alpha_beta_and_empty_rows(cuda, algo):
    import torch
    rng = np.random.default_rng(0)
    n = 1000
    lens = rng.integers(0, 4, n)
    lens[:50] = 0
    lens[-50:] = 0
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    va = rng.standard_normal(ci.size)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, n)
    ref = 2.5 * pyoracle.spmv_f64(rp, ci, va, x) - 0.5 * y0
    d = _dev(cuda, rp, ci, va, x)
    y = torch.from_numpy(y0.copy()).to(cuda)
    bsp.csr_spmv(*d, y=y, alpha=2.5, beta=-0.5, algo=algo)
    tol = 2.5 * pyoracle.spmv_tolerance(rp, ci, va, x) + 4 * 2.0 ** -53 * (np.abs(ref) + 1)
    _within(y.cpu().numpy(), ref, tol)


def test_empty_matrix(cuda):
    import torch
    rp = torch.zeros(101, dtype=torch.int32, device=cuda)
    ci = torch.zeros(0, dtype=torch.int32, device=cuda)
    va = torch.zeros(0, dtype=torch.float64, device=cuda)
    x = torch.ones(100, dtype=torch.float64, device=cuda)
    for algo in ("vector", "merge", "scalar", "stream"):
        y = torch.full((100,), 7.0, dtype=torch.float64, device=cuda)
        bsp.csr_spmv(rp, ci, va, x, y=y, algo=algo)
        assert torch.all(y == 0)


def test_merge_workspace_too_small_is_rejected(cuda):
    import torch
    A = bsp.gen_laplace2d(32, 32)
    d = _dev(cuda, A.rowptr, A.colidx, A.values, np.ones(A.cols))
    ws = torch.empty(8, dtype=torch.uint8, device=cuda)
    with pytest.raises(bsp.BspError):
        bsp.csr_spmv_merge(*d, workspace=ws)
