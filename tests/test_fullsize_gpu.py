"""Parity at the benchmark sizes: every benchmarked workload, at the size and
seeds bench.py runs, checked against the CPU oracle with the same bounds the
small tests use.

* SpMV (FP64): per row |y - y_oracle| <= 2*gamma_L*sum_j |a_ij x_j| with
  gamma_L = L*u/(1 - L*u), u = 2^-53, L = row length + 1 (any summation
  order; `pyoracle.spmv_tolerance`).  Oracle: `ref_spmv_fp64`,
  src/ref.cpp:26-37.
* Conversions: bit-exact with the oracle's restatement of the reference's
  converters (DASP packing, src/dasp.cu:814-1482).
* CG: ||b - A x|| / ||b|| <= 1e-10 recomputed with the oracle's FP64 SpMV,
  every storage mode.
* SpMM (FP16/BF16 inputs, FP32 accumulation): products of two 16-bit floats
  are exact in FP32, so |C - C_fp64| <= 2*gamma_L*(|A||B|), u = 2^-24,
  L = row length + 2, against the FP64 SpMM of the same rounded inputs; and
  the relative error against the FP64 SpMM of the unrounded inputs <= 1e-2.
  The oracle covers a stated row sample (every 256th row plus the 32
  longest rows), since the full FP64 SpMM at N = 256 would take minutes.
* Batch: all 512 matrices, 1 and 8 right-hand sides, FP64 and FP32.
"""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu

SEED = 20261203 + 1     # the headline's seed; the other workloads use SEED + k as bench.py does


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _assert_within(y, ref, tol, what):
    bad = np.abs(y - ref) > tol
    assert not bad.any(), (f"{what}: {int(bad.sum())} rows outside the bound, first {np.flatnonzero(bad)[:5]}, "
                           f"worst excess {float(np.max((np.abs(y - ref) - tol)[bad]))}")


# ---------------------------------------------------------------------------
# C1: CSR FP64 on the 2-D 5-point Laplacian 512 x 512

@pytest.mark.parametrize("algo", ["auto", "vector", "merge", "scalar"])
def test_c1_csr_laplace512(cuda, algo):
    A = bsp.gen_laplace2d(512, 512)
    x = bsp.gen_uniform(A.cols, SEED + 10)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    y = bsp.csr_spmv(rp, ci, va, xx, algo=algo).cpu().numpy()
    if algo == "scalar":
        assert np.array_equal(y, ref)
    else:
        _assert_within(y, ref, pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x), algo)


# ---------------------------------------------------------------------------
# C2a / C2b: the headline matrix (27-point stencil 64^3 x 4 dof), 4x4 and 8x8

@pytest.fixture(scope="module")
def stencil():
    A = bsp.gen_stencil27(64, 4, SEED)
    x = bsp.gen_uniform(A.cols, SEED + 1)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    return A, x, ref, tol


@pytest.mark.parametrize("bs,algo", [(4, "auto"), (4, "dmma"), (8, "auto")])
def test_c2_stencil64_bsr(cuda, stencil, bs, algo):
    """The benchmarked call (4x4, FFMA kernel) and the DMMA kernel, plus the
    8x8 re-blocking (fill 50.5%): within the FP64 bound of ref_spmv_fp64 on
    all 1,048,576 rows; the conversion's block count is the stencil's
    closed form."""
    import torch
    A, x, ref, tol = stencil
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
    del rp, ci, va
    if bs == 4:
        assert M.blc_num == 190 ** 3 and A.nnz == 16 * 190 ** 3
    else:
        assert M.blc_num == 94 * 190 ** 2
    y = M.spmv(xx, algo=algo).cpu().numpy()
    _assert_within(y, ref, tol, f"bsr{bs} {algo}")
    # y = alpha*A*x + beta*y on the same call
    y0 = torch.from_numpy(ref).to(cuda)
    y2 = M.spmv(xx, y0, alpha=2.0, beta=-1.0, algo=algo).cpu().numpy()
    _assert_within(y2, ref, 2 * tol + 4 * 2.0 ** -53 * np.abs(ref), f"bsr{bs} {algo} alpha/beta")
    M.free()
    torch.cuda.synchronize()


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
def test_c2_stencil64_scaled_16bit(cuda, stencil, dtype):
    """The headline matrix stored as FP16/BF16 with one power-of-two scale
    per 4x4 block: the quantized arrays bit-exact with the oracle's
    restatement of the format, the FP32-accumulated SpMV within
    2*gamma_L(2^-24) * sum |a x| (L = row length + 3) of the FP64 product of
    the dequantized matrix, and within that plus the quantization error
    (sum |q 2^e - a| |x|, at most 2^-11 for FP16 / 2^-8 for BF16 of sum |a x|
    on these N(0,1) blocks) of ref_spmv_fp64 on the FP64 matrix."""
    A, x, ref, tol = stencil
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=4)
    del rp, ci, va
    S = M.scaled(dtype)
    src = M.arrays()
    M.free()
    got = S.arrays()
    key, val, bad = pyoracle.bsr_scale(src["blcIdx"], src["blcVal"], 4, dtype)
    assert bad == 0 and np.array_equal(got["blcKey"], key) and np.array_equal(got["blcVal"], val)
    del got
    y = S.spmv(xx).cpu().numpy()
    S.free()
    deq = pyoracle.bsr_unscale(key, val, 4, dtype)
    del key, val
    yq, ayq = pyoracle.bsr_spmv_f64(A.rows, src["blcPtr"], src["blcIdx"], deq, 4, x)
    deq -= src["blcVal"]
    _, qerr = pyoracle.bsr_spmv_f64(A.rows, src["blcPtr"], src["blcIdx"], deq, 4, x)
    del deq
    L = np.diff(A.rowptr).astype(np.float64) + 3.0
    u = 2.0 ** -24
    tq = 2.0 * (L * u / (1.0 - L * u)) * ayq + 1e-300
    _assert_within(y, yq, tq, f"scaled {dtype} vs dequantized")
    # quantization error sum_j |q 2^e - a| |x_j|, exact from the oracle's arrays;
    # for normal values it is below 2^-11 (FP16) / 2^-8 (BF16) of sum |a x|
    quant = {"f16": 2.0 ** -11, "bf16": 2.0 ** -8}[dtype]
    absrow = pyoracle.abs_rowsum(A.rowptr, A.colidx, A.values, x)
    assert np.all(qerr <= 1.001 * quant * absrow + 1e-300)
    _assert_within(y, ref, tq + tol + 1.001 * qerr + 2.0 ** -50 * ayq, f"scaled {dtype} vs ref_spmv_fp64")


@pytest.mark.parametrize("bs", [4, 8])
def test_c2c_random_block_fill(cuda, bs):
    """16 random block columns per block row, per-block fill U[30%, 100%]."""
    nbr = 262144 if bs == 4 else 131072
    A = bsp.gen_random_bsr(nbr, bs, 16, 0.3, 1.0, SEED + 11)
    x = bsp.gen_uniform(A.cols, SEED + 12)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    M = bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)
    assert M.blc_num == nbr * 16
    y = M.spmv(xx).cpu().numpy()
    _assert_within(y, ref, pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x), f"random bsr{bs}")
    M.free()


# ---------------------------------------------------------------------------
# C2d: DASP on the 2M-row power-law matrix (Zipf 2.0, rows capped at 10k)

DASP_ARRS = ("long_val", "long_cid", "long_ptr_warp", "reg_val", "reg_cid", "block_ptr", "irreg_val", "irreg_cid",
             "irreg_rpt", "short_val", "short_cid", "order_rid")
DASP_INTS = ("row_long", "row_block", "blocknum", "short_row_1", "common_13", "short_row_34", "short_row_2",
             "offset_reg", "offset_short1", "offset_short13", "offset_short34", "offset_short22",
             "fill0_nnz_short13", "fill0_nnz_short34")


def test_c2d_dasp_powerlaw_2m(cuda):
    import torch
    A = bsp.gen_powerlaw(1 << 21, 2.0, 10000, SEED + 13)
    x = bsp.gen_uniform(A.cols, SEED + 14)
    rp, ci, va, xx = _dev(cuda, A.rowptr, A.colidx, A.values, x)
    D = bsp.csr2dasp(rp, ci, va, rows=A.rows, cols=A.cols)
    o = pyoracle.dasp_pack(A.rowptr, A.colidx, A.values)
    got = D.arrays()
    for k in DASP_ARRS:
        assert np.array_equal(got[k], o[k]), k
    for k in DASP_INTS:
        assert getattr(D, k) == o[k], k
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    y = torch.empty(A.rows, dtype=torch.float64, device=cuda)
    for _ in range(2):   # the second call reuses the long-row arrival counters
        D.spmv(xx, y)
        _assert_within(y.cpu().numpy(), ref, tol, "dasp")
    yp = D.spmv(xx, permuted=True).cpu().numpy()
    order = got["order_rid"]
    _assert_within(yp, ref[order], tol[order], "dasp permuted")
    D.free()


# ---------------------------------------------------------------------------
# C3: CG on the 7-point Poisson 128^3, every storage mode, to 1e-10

@pytest.fixture(scope="module")
def poisson128():
    A = bsp.gen_poisson3d(128)
    b = bsp.gen_uniform(A.rows, SEED + 3)
    return A, b


@pytest.fixture(scope="module")
def poisson128_fp64_solution(poisson128, cuda):
    A, b = poisson128
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    S = bsp.CgSolver(rp, ci, va, mode="fp64", tol=1e-10)
    x, res = S.solve(bb)
    S.close()
    return x.cpu().numpy(), res


@pytest.mark.parametrize("mode", ["fp64", "f32", "f16", "bf16"])
def test_c3_cg_poisson128(cuda, poisson128, poisson128_fp64_solution, mode):
    A, b = poisson128
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10)
    x, res = S.solve(bb)
    S.close()
    x = x.cpu().numpy()
    assert res["converged"] == 1 and res["rel_residual"] <= 1e-10
    # the solver's own FP64 residual, recomputed on the CPU by the oracle
    assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, x) <= 1.0001e-10
    x64, r64 = poisson128_fp64_solution
    # same solution as the FP64 solve: ||dx|| <= cond(A) * 2e-10 * ||x||, cond ~ 6.7e3
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 2e-6
    # the reliable updates keep the mixed modes at the FP64 iteration count (+2%)
    assert res["iterations"] <= 1.02 * r64["iterations"] + 2


# ---------------------------------------------------------------------------
# C4: SpMM on the power-law graph (n = 2^20, Zipf 1.8, mean degree 32)

@pytest.fixture(scope="module")
def graph():
    A = bsp.gen_graph(1 << 20, 1.8, 32, SEED + 4)
    lens = np.diff(A.rowptr)
    sample = np.union1d(np.arange(0, A.rows, 256), np.argsort(lens, kind="stable")[-32:]).astype(np.int64)
    return A, sample


def _sample_csr(A, rows):
    """Sub-CSR of `rows`, columns renumbered into the distinct columns used."""
    lens = np.diff(A.rowptr)[rows]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    idx = np.concatenate([np.arange(A.rowptr[r], A.rowptr[r + 1]) for r in rows])
    cols, inv = np.unique(A.colidx[idx], return_inverse=True)
    return rp, inv.astype(np.int32), idx, cols


@pytest.mark.parametrize("name", ["f16", "bf16"])
@pytest.mark.parametrize("N", [32, 128, 256])
def test_c4_spmm_graph_1m(cuda, graph, name, N):
    import torch
    A, sample = graph
    tdt = {"f16": torch.float16, "bf16": torch.bfloat16}[name]
    rp, ci, v64 = _dev(cuda, A.rowptr, A.colidx, A.values)
    v = v64.to(tdt)
    g = torch.Generator(device="cpu").manual_seed(N)
    B64 = torch.rand(A.cols, N, generator=g, dtype=torch.float64) * 2 - 1
    B = B64.to(tdt).to(cuda)
    P = bsp.SpmmPlan(rp, ci, v, cols=A.cols, chunk=256)
    C1 = P.spmm(B)
    C2 = bsp.spmm_csr(rp, ci, v, B)
    assert torch.equal(C1, P.spmm(B)), "planned SpMM is not deterministic"
    srp, sci, idx, cols = _sample_csr(A, sample)
    Bs = B[torch.from_numpy(cols).to(cuda)].double().cpu().numpy()
    vq = v.double().cpu().numpy()[idx]
    Cref, absC = pyoracle.spmm_f64(srp, sci, vq, Bs)
    L = (np.diff(srp).astype(np.float64) + 2.0)[:, None]
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1.0 - L * u)) * absC + 1e-30
    rows_d = torch.from_numpy(sample).to(cuda)
    for what, Cm in (("planned", C1), ("plan-free", C2)):
        got = Cm[rows_d].double().cpu().numpy()
        bad = np.abs(got - Cref) > tol
        assert not bad.any(), f"{what}: {int(bad.sum())} entries outside the FP32 accumulation bound"
    # against the FP64 product of the unrounded values and B (the 1e-2 target)
    Cx, _ = pyoracle.spmm_f64(srp, sci, A.values[idx], B64[torch.from_numpy(cols)].numpy())
    got = C1[rows_d].double().cpu().numpy()
    assert np.linalg.norm(got - Cx) / np.linalg.norm(Cx) <= 1e-2
    P.free()


# ---------------------------------------------------------------------------
# C5: 512 matrices in one persistent launch

@pytest.fixture(scope="module")
def batch512():
    return bsp.gen_batch(512, SEED + 6)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("nrhs", [1, 8])
def test_c5_batch_512(cuda, batch512, dtype, nrhs):
    import torch
    mats = batch512
    tdt = torch.float64 if dtype == "f64" else torch.float32
    unit = 2.0 ** -53 if dtype == "f64" else 2.0 ** -24
    g = torch.Generator(device="cpu").manual_seed(nrhs)
    d, host = [], []
    for m in mats:
        vals = torch.from_numpy(m.values).to(tdt)
        x = (torch.rand((m.cols, nrhs) if nrhs > 1 else (m.cols,), generator=g, dtype=torch.float64) * 2 - 1).to(tdt)
        y = torch.full((m.rows, nrhs) if nrhs > 1 else (m.rows,), float("nan"), dtype=tdt, device=cuda)
        d.append((*_dev(cuda, m.rowptr, m.colidx), vals.to(cuda), x.to(cuda), y))
        host.append((vals.double().numpy(), x.double().numpy()))
    P = bsp.BatchPlan(d, nrhs=nrhs, tune=1)
    assert P.stats()["nnz"] == sum(int(m.rowptr[-1]) for m in mats)
    P.run()
    torch.cuda.synchronize()
    first = []
    for m, dd, (vals, x) in zip(mats, d, host):
        got = dd[4].double().cpu().numpy()
        first.append(got)
        if nrhs == 1:
            want = pyoracle.spmv_f64(m.rowptr, m.colidx, vals, x)
            tol = pyoracle.spmv_tolerance(m.rowptr, m.colidx, vals, x, unit)
        else:
            want, absC = pyoracle.spmm_f64(m.rowptr, m.colidx, vals, x)
            L = (np.diff(m.rowptr).astype(np.float64) + 1.0)[:, None]
            tol = 2.0 * (L * unit / (1 - L * unit)) * absC + np.finfo(np.float64).tiny
        assert np.all(np.abs(got - want) <= tol)
    # a replay of the captured launch gives the same bits
    for dd in d:
        dd[4].fill_(float("nan"))
    P.run()
    torch.cuda.synchronize()
    for got, dd in zip(first, d):
        assert np.array_equal(got, dd[4].double().cpu().numpy())
    P.close()
