"""The allocation-free merge-path SpMV (bsp_csr_spmv_merge_f64_noalloc),
called through the C ABI, against the existing merge-path entry point
(bsp_csr_spmv_merge_f64 with a caller-provided workspace).

It exists for hosts that may not allocate device memory while they run (all
memory handed to their own pool at start-up, or loops that must not call
cudaMalloc/cudaFree).  Two calls in a row check that the shared in-library
workspace carries nothing wrong from one call into the next.  This file is
collected last so that a run stopping at its first failure has run every
other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import benchsp_b200 as bsp
from benchsp_b200 import _lib
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _noalloc(L, rows, cols, rp, ci, va, x, y, alpha, beta, stream):
    return L.bsp_csr_spmv_merge_f64_noalloc(rows, cols, ci.numel(), _p(rp), _p(ci), _p(va), _p(x), _p(y),
                                            alpha, beta, stream)


@pytest.mark.parametrize("kind", ["powerlaw_long_rows", "laplace"])
def test_noalloc_matches_workspace_entry_point_on_two_calls(cuda, kind):
    import torch
    L = bsp.lib()
    A = (bsp.gen_powerlaw(150000, 1.6, 60000, 91) if kind == "powerlaw_long_rows"
         else bsp.gen_laplace2d(512, 512))
    rp, ci, va = (torch.from_numpy(a).to(cuda) for a in (A.rowptr, A.colidx, A.values))
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ws = torch.empty(bsp.csr_merge_workspace_bytes(A.rows, A.nnz), dtype=torch.uint8, device=cuda)
    for call, (seed, alpha, beta) in enumerate([(1, 1.0, 0.0), (2, -0.5, 2.0)]):
        x_h = bsp.gen_uniform(A.cols, seed)
        y0_h = bsp.gen_uniform(A.rows, seed + 10)
        x = torch.from_numpy(x_h).to(cuda)
        y_ref = torch.from_numpy(y0_h).to(cuda)
        y_new = torch.from_numpy(y0_h).to(cuda)
        _lib.check(L.bsp_csr_spmv_merge_f64(A.rows, A.cols, A.nnz, _p(rp), _p(ci), _p(va), _p(x), _p(y_ref),
                                            alpha, beta, _p(ws), ws.numel(), stream))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _lib.check(_noalloc(L, A.rows, A.cols, rp, ci, va, x, y_new, alpha, beta, stream))
        torch.cuda.synchronize()
        if call > 0:
            # after the first call has set the array up, a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before, "the allocation-free call changed free memory"
        a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
        # the same kernels in the same order as the workspace entry point: the same bits
        assert np.array_equal(a, b), f"call {call}"
        # against the oracle: the per-row rounding bound (scaled by |alpha|)
        # plus the rounding of alpha*(A x) + beta*y
        ax = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x_h)
        tol = abs(alpha) * pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x_h) + \
            4 * 2.0 ** -53 * (np.abs(alpha * ax) + np.abs(beta * y0_h))
        ref = alpha * ax + beta * y0_h
        assert np.all(np.abs(a - ref) <= 2 * tol), f"call {call} vs oracle"


def test_noalloc_rejects_inputs_over_its_limit(cuda):
    import torch
    L = bsp.lib()
    dummy = torch.zeros(1, dtype=torch.float64, device=cuda)
    st = L.bsp_csr_spmv_merge_f64_noalloc(60000000, 60000000, 10000000, _p(dummy), _p(dummy), _p(dummy),
                                          _p(dummy), _p(dummy), 1.0, 0.0, None)
    assert st == _lib.BSP_ERR_INVALID
    assert b"allocation-free limit" in L.bsp_last_error()
