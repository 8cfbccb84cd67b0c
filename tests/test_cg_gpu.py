"""CG on the GPU: FP64 and mixed precision (FP32 / per-group-scaled FP16 and
BF16 storage, FP64 refinement) reach ||b - A x|| / ||b|| <= 1e-10, checked
with the CPU oracle's FP64 SpMV, and agree with the CPU FP64 CG oracle."""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def _permuted_laplace(nx, seed):
    """A symmetric permutation of a 2-D Laplacian: SPD, and with nx*nx > 32768
    rows some |col - row| exceed the int16 offset range."""
    import scipy.sparse as sp
    A = bsp.gen_laplace2d(nx, nx)
    M = sp.csr_matrix((A.values, A.colidx, A.rowptr), shape=(A.rows, A.rows))
    perm = np.random.default_rng(seed).permutation(A.rows)
    M = M[perm][:, perm].tocsr()
    M.sort_indices()
    return bsp.HostCSR(A.rows, A.rows, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.copy())


def _ragged_laplace(nx):
    """2-D Laplacian plus symmetric couplings (-0.1) from every 97th row to
    the rows 100, 200, ..., 1000 after it, diagonal raised to keep it
    diagonally dominant: SPD, offsets within int16, and SELL-32 slices of
    uneven length (padding all to the longest would cost far more than 1/32
    extra storage, so the low-precision copy keeps per-slice lengths)."""
    import scipy.sparse as sp
    A = bsp.gen_laplace2d(nx, nx)
    n = A.rows
    M = sp.csr_matrix((A.values, A.colidx, A.rowptr), shape=(n, n)).tolil()
    for i in range(0, n, 97):
        for d in range(100, 1001, 100):
            if i + d < n:
                M[i, i + d] = M[i + d, i] = -0.1
                M[i, i] += 0.1
                M[i + d, i + d] += 0.1
    M = M.tocsr()
    M.sort_indices()
    return bsp.HostCSR(n, n, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.copy())


@pytest.mark.parametrize("mode", ["f32", "f16", "bf16"])
def test_cg_mixed_uneven_slices(cuda, mode):
    A = _ragged_laplace(120)
    lens = np.zeros(-(-A.rows // 32) * 32, np.int64)
    lens[:A.rows] = np.diff(A.rowptr)
    sl = lens.reshape(-1, 32).max(axis=1)
    assert sl.size * 32 * sl.max() > 32 * sl.sum() * 33 // 32      # per-slice lengths are kept
    b = bsp.gen_uniform(A.rows, 12)
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10)
    x, res = S.solve(bb)
    S.close()
    x = x.cpu().numpy()
    assert res["converged"] == 1 and res["delta16"] == 1
    assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, x) <= 2e-10
    xr, _ = pyoracle.cg(A.rowptr, A.colidx, A.values, b, 1e-12)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-7


@pytest.mark.parametrize("mode", ["fp64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("kind", ["poisson24", "permuted_laplace"])
def test_cg_reaches_1e10(cuda, mode, kind):
    A = bsp.gen_poisson3d(24) if kind == "poisson24" else _permuted_laplace(200, 4)
    b = bsp.gen_uniform(A.rows, 11)
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    S = bsp.CgSolver(rp, ci, va, mode=mode, tol=1e-10)
    x, res = S.solve(bb)
    x = x.cpu().numpy()
    assert res["converged"] == 1 and res["rel_residual"] <= 1e-10
    assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, x) <= 2e-10
    if mode != "fp64":
        assert res["reliable_updates"] >= 2
        assert res["delta16"] == (1 if kind == "poisson24" else 0)
    xr, _ = pyoracle.cg(A.rowptr, A.colidx, A.values, b, 1e-12)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-7


def test_cg_repeated_solves_and_initial_guess(cuda):
    import torch
    A = bsp.gen_poisson3d(16)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    S = bsp.CgSolver(rp, ci, va, mode="f16")
    for seed in (1, 2):
        b = bsp.gen_uniform(A.rows, seed)
        x, res = S.solve(_dev(cuda, b)[0])
        assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, x.cpu().numpy()) <= 2e-10
    # starting from the solution: no iterations needed
    x2, res2 = S.solve(_dev(cuda, b)[0], x.clone())
    assert res2["iterations"] == 0 and res2["converged"] == 1


def test_cg_not_converged_is_reported(cuda):
    A = bsp.gen_poisson3d(16)
    b = bsp.gen_uniform(A.rows, 5)
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    S = bsp.CgSolver(rp, ci, va, mode="fp64", max_iters=4, check_every=2)
    with pytest.raises(bsp.BspError):
        S.solve(bb)
    x, res = S.solve(bb, raise_on_stall=False)
    assert res["converged"] == 0 and res["rel_residual"] > 1e-10


def test_cg_without_graphs_matches(cuda):
    A = bsp.gen_poisson3d(12)
    b = bsp.gen_uniform(A.rows, 9)
    rp, ci, va, bb = _dev(cuda, A.rowptr, A.colidx, A.values, b)
    x1, r1 = bsp.CgSolver(rp, ci, va, mode="f16", use_graphs=True).solve(bb)
    x2, r2 = bsp.CgSolver(rp, ci, va, mode="f16", use_graphs=False).solve(bb)
    assert r1["iterations"] == r2["iterations"]
    assert np.array_equal(x1.cpu().numpy(), x2.cpu().numpy())
