"""FP16/BF16 BSR with one power-of-two scale per block (bsp_bsr_scaled).

The quantized arrays must equal the oracle's restatement of the format bit
for bit (oracle/oracle_formats.c: orc_bsr_scale).  The SpMV computes in FP32:
x rounded to FP32 (relative error u = 2^-24) and scaled by the block's 2^e
(exact), FMA chains and shuffle sums in FP32.  Against the FP64 product of the
dequantized matrix (exact values q * 2^e) it is therefore within
2*gamma_L*sum_j |a_ij x_j|, gamma_L = L*u/(1 - L*u), L = stored entries in the
row + 3, for any summation order, plus the rounding of alpha*s + beta*y in the
type of y.  Against the unquantized FP64 matrix the quantization adds
sum_j |q_ij 2^e - a_ij| |x_j|, computed exactly from the oracle's arrays; each
quantized entry is within half a unit in the last place of the 16-bit type
at the block's scale (relative 2^-11 for FP16 and 2^-8 for BF16, or the
type's smallest step times 2^e for entries that fall below its normal range
at that scale; oracle test in tests/test_oracle.py).
"""
import ctypes as C

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _wide_range(A, seed):
    """Row scales 10^k, k in [-20, 20]: blocks far apart in magnitude."""
    rng = np.random.default_rng(seed)
    s = 10.0 ** rng.integers(-20, 21, A.rows)
    v = A.values * np.repeat(s, np.diff(A.rowptr))
    return bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, v)


MATS = {
    "stencil6": lambda: bsp.gen_stencil27(6, 4, 3),
    "random_bsr4": lambda: bsp.gen_random_bsr(300, 4, 16, 0.3, 1.0, 4),
    "random_bsr8": lambda: bsp.gen_random_bsr(150, 8, 12, 0.3, 1.0, 5),
    "powerlaw_ragged": lambda: bsp.gen_powerlaw(5003, 1.8, 900, 6),
    "wide_range": lambda: _wide_range(bsp.gen_stencil27(5, 4, 7), 8),
}


def _build(cuda, A, bs):
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    return bsp.csr2bsr(rp, ci, va, rows=A.rows, cols=A.cols, bs=bs)


def _reference(A, M, arr, dtype, x):
    """(FP64 product of the dequantized matrix, its |a||x| row sums, the
    unquantized FP64 product, the row sums of |quantization error| |x|)."""
    bs = M.bs
    deq = pyoracle.bsr_unscale(arr["blcKey"], arr["blcVal"], bs, dtype)
    src = M.arrays()
    y, ay = pyoracle.bsr_spmv_f64(A.rows, src["blcPtr"], src["blcIdx"], deq, bs, x)
    y64, _ = pyoracle.bsr_spmv_f64(A.rows, src["blcPtr"], src["blcIdx"], src["blcVal"], bs, x)
    _, qerr = pyoracle.bsr_spmv_f64(A.rows, src["blcPtr"], src["blcIdx"], deq - src["blcVal"], bs, x)
    return y, ay, y64, qerr


def _tol(A, M, ay):
    blocks = np.diff(M.arrays()["blcPtr"]).astype(np.float64)
    L = np.repeat(blocks * M.bs, M.bs)[:A.rows] + 3.0
    return 2.0 * (L * U32 / (1.0 - L * U32)) * ay + 1e-300


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
@pytest.mark.parametrize("bs", [4, 8])
@pytest.mark.parametrize("name", list(MATS))
def test_scaled_arrays_bit_exact_and_spmv_within_bound(cuda, name, bs, dtype):
    A = MATS[name]()
    M = _build(cuda, A, bs)
    S = M.scaled(dtype)
    arr = S.arrays()
    src = M.arrays()
    key, val, bad = pyoracle.bsr_scale(src["blcIdx"], src["blcVal"], bs, dtype)
    assert bad == 0
    assert np.array_equal(arr["blcKey"], key) and np.array_equal(arr["blcVal"], val)
    assert np.array_equal(arr["blcPtr"], src["blcPtr"])
    x = bsp.gen_uniform(A.cols, 21)
    y_ref, ay, y64, qerr = _reference(A, M, arr, dtype, x)
    import torch
    xx = _dev(cuda, x)[0]
    y = S.spmv(xx).cpu().numpy()
    tol = _tol(A, M, ay)
    assert np.all(np.abs(y - y_ref) <= tol)
    # against the FP64 matrix: the FP32 bound plus the quantization error
    # (with a margin for the FP64 rounding of the two reference products)
    assert np.all(np.abs(y - y64) <= tol + 1.001 * qerr + 2.0 ** -50 * (ay + np.abs(y64)) + 1e-300)
    # FP32 x and y
    y32 = S.spmv(xx.float()).cpu().numpy().astype(np.float64)
    x32 = x.astype(np.float32).astype(np.float64)
    y_ref32, ay32, _, _ = _reference(A, M, arr, dtype, x32)
    assert np.all(np.abs(y32 - y_ref32) <= _tol(A, M, ay32) + U32 * np.abs(y_ref32))
    # alpha, beta
    y0 = torch.from_numpy(bsp.gen_uniform(A.rows, 22)).to(cuda)
    yb = S.spmv(xx, y0.clone(), alpha=-1.5, beta=0.25).cpu().numpy()
    want = -1.5 * y_ref + 0.25 * y0.cpu().numpy()
    assert np.all(np.abs(yb - want) <= 1.5 * tol + 4 * 2.0 ** -53 * (np.abs(want) + 1))
    S.free()
    M.free()


@pytest.mark.parametrize("bs,lanes,unroll", [(4, 4, 1), (4, 8, 1), (4, 16, 1), (4, 32, 1), (4, 4, 2), (4, 8, 2),
                                             (4, 16, 2), (8, 4, 1), (8, 8, 1), (8, 16, 1), (8, 32, 1), (8, 8, 2),
                                             (8, 16, 2)])
def test_scaled_every_kernel_shape(cuda, bs, lanes, unroll):
    A = bsp.gen_powerlaw(4001, 1.6, 1500, 12)   # long and empty block rows, cols % 8 != 0
    M = _build(cuda, A, bs)
    S = M.scaled("f16")
    x = bsp.gen_uniform(A.cols, 3)
    y_ref, ay, _, _ = _reference(A, M, S.arrays(), "f16", x)
    xx = _dev(cuda, x)[0]
    y = S.spmv(xx, lanes=lanes, unroll=unroll).cpu().numpy()
    assert np.all(np.abs(y - y_ref) <= _tol(A, M, ay))
    # x not 32-byte aligned: the kernel's scalar x path
    import torch
    xbig = torch.zeros(A.cols + 1, dtype=torch.float64, device=cuda)
    xbig[1:] = xx
    y2 = S.spmv(xbig[1:], lanes=lanes, unroll=unroll).cpu().numpy()
    assert np.array_equal(y, y2)
    S.free()
    M.free()


def test_scaled_is_deterministic_and_rejects_bad_input(cuda):
    import torch
    A = bsp.gen_stencil27(7, 4, 9)
    M = _build(cuda, A, 4)
    S = M.scaled("bf16")
    xx = _dev(cuda, bsp.gen_uniform(A.cols, 1))[0]
    assert torch.equal(S.spmv(xx), S.spmv(xx))
    with pytest.raises(ValueError):
        S.spmv(xx.to(torch.float16))
    S.free()
    M.free()
    # a value beyond the 16-bit range after the block's clamped scale
    v = A.values.copy()
    v[5] = 1e300
    M2 = _build(cuda, bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, v), 4)
    with pytest.raises(bsp.BspError):
        M2.scaled("f16")
    v[5] = np.inf
    M3 = _build(cuda, bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, v), 4)
    with pytest.raises(bsp.BspError):
        M3.scaled("bf16")
    M2.free()
    M3.free()
    st = bsp.lib().bsp_bsr_scaled_create(C.byref(M.desc), 0, C.byref(bsp._lib.BspBsrScaled()), None)
    assert st == bsp._lib.BSP_ERR_INVALID
