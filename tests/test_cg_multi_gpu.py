"""CG with several right-hand sides (bsp_cg_solve_multi): every column
reaches 1e-10 (checked with the oracle's FP64 SpMV), matches the oracle's
FP64 CG / PCG solution, needs the iteration count of a single solve; groups
of more than 8 columns, strided B / X, an exact initial guess, and the plans
it rejects."""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


@pytest.mark.parametrize("k", [1, 3, 8, 11])
@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_multi_rhs_matches_single_solves(cuda, k, precond):
    import torch
    A = bsp.gen_diffusion3d(14, 2.0, 5) if precond == "jacobi" else bsp.gen_poisson3d(14)
    rng = np.random.default_rng(k)
    Bh = rng.uniform(-1, 1, (A.rows, k))
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    S = bsp.CgSolver(rp, ci, va, mode="fp64", precond=precond)
    X, rel, res = S.solve_multi(torch.from_numpy(Bh).to(cuda))
    Xh = X.cpu().numpy()
    assert res["converged"] == 1 and np.all(rel <= 1e-10) and res["rel_residual"] == rel.max()
    its = []
    for j in range(k):
        b = np.ascontiguousarray(Bh[:, j])
        assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, Xh[:, j]) <= 2e-10
        if precond == "none":
            xr, it = pyoracle.cg(A.rowptr, A.colidx, A.values, b, 1e-10)
        else:
            xr, it = pyoracle.pcg(A.rowptr, A.colidx, A.values, b, 1, 1e-10)
        its.append(it)
        xs, _ = pyoracle.cg(A.rowptr, A.colidx, A.values, b, 1e-13) if precond == "none" else \
            pyoracle.pcg(A.rowptr, A.colidx, A.values, b, 1, 1e-13)
        assert np.linalg.norm(Xh[:, j] - xs) / np.linalg.norm(xs) < 1e-8
    assert res["iterations"] <= max(its) + 16      # chunks of 16 between checks
    S.close()


def test_strided_arrays_and_exact_guess(cuda):
    import torch
    A = bsp.gen_poisson3d(10)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    S = bsp.CgSolver(rp, ci, va, mode="fp64")
    wide = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (A.rows, 7))).to(cuda)
    B = wide[:, 1:6]                                   # ldb = 7, k = 5
    Xw = torch.zeros(A.rows, 9, dtype=torch.float64, device=cuda)
    X = Xw[:, 2:7]                                     # ldx = 9
    X, rel, res = S.solve_multi(B, X)
    assert res["converged"] == 1
    assert torch.count_nonzero(Xw[:, :2]) == 0 and torch.count_nonzero(Xw[:, 7:]) == 0
    Bh = B.cpu().numpy()
    for j in range(5):
        assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, np.ascontiguousarray(Bh[:, j]),
                                     X[:, j].cpu().numpy()) <= 2e-10
    X2, rel2, res2 = S.solve_multi(B, X.clone())      # start from the solution
    assert res2["iterations"] == 0 and res2["converged"] == 1
    S.close()


def test_unsupported_plans(cuda):
    import torch
    A = bsp.gen_poisson3d(6)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    B = torch.ones(A.rows, 2, dtype=torch.float64, device=cuda)
    for kw in ({"mode": "f16"}, {"mode": "fp64", "precond": "block_jacobi"}):
        S = bsp.CgSolver(rp, ci, va, **kw)
        with pytest.raises(bsp.BspError) as e:
            S.solve_multi(B)
        assert e.value.status == bsp._lib.BSP_ERR_UNSUPPORTED
        S.close()
