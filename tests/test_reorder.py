"""Reverse Cuthill-McKee reordering and symmetric permutation: valid
permutations, bandwidth as small as scipy's RCM, P A P^T exact, components
and edge cases on the host; on the GPU the device forms agree with the host
forms and reordering a scrambled stencil raises the SMaT 16x16 tile fill."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

import benchsp_b200 as bsp


def _scramble(A, seed):
    M = sp.csr_matrix((A.values, A.colidx, A.rowptr), shape=(A.rows, A.cols))
    p = np.random.default_rng(seed).permutation(A.rows)
    Mp = M[p][:, p].tocsr()
    Mp.sort_indices()
    return bsp.HostCSR(A.rows, A.cols, Mp.indptr.astype(np.int32), Mp.indices.astype(np.int32), Mp.data.copy())


def _bandwidth(A):
    r = np.repeat(np.arange(A.rows), np.diff(A.rowptr))
    return int(np.abs(A.colidx - r).max()) if A.nnz else 0


def _scipy(A):
    return sp.csr_matrix((A.values, A.colidx, A.rowptr), shape=(A.rows, A.cols))


@pytest.mark.parametrize("kind", ["stencil", "banded", "laplace"])
def test_rcm_bandwidth_and_exact_permutation(kind):
    A = {"stencil": lambda: bsp.gen_stencil27(12, 2, 1), "banded": lambda: bsp.gen_banded(5000, 9, 2),
         "laplace": lambda: bsp.gen_laplace2d(70, 40)}[kind]()
    B = _scramble(A, 7)
    perm = bsp.reorder_rcm_host(B.rowptr, B.colidx)
    assert np.array_equal(np.sort(perm), np.arange(B.rows))
    R = bsp.permute_csr_host(B, perm)
    ref = _scipy(B)[perm][:, perm].tocsr()
    ref.sort_indices()
    assert np.array_equal(R.rowptr, ref.indptr) and np.array_equal(R.colidx, ref.indices)
    assert np.array_equal(R.values, ref.data)
    ps = reverse_cuthill_mckee(_scipy(B), symmetric_mode=True).astype(np.int32)
    assert _bandwidth(R) <= 1.05 * _bandwidth(bsp.permute_csr_host(B, ps)) + 1
    assert _bandwidth(R) < _bandwidth(B) / 4


def test_rcm_components_isolated_rows_and_unsymmetric_pattern():
    # two components, an isolated vertex, an unsymmetric entry
    dense = np.zeros((9, 9))
    for i, j in [(0, 1), (1, 2), (2, 0), (4, 5), (5, 6), (6, 7), (7, 4), (8, 5)]:
        dense[i, j] = 1.0
    np.fill_diagonal(dense, 2.0)
    M = sp.csr_matrix(dense)
    A = bsp.HostCSR(9, 9, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.copy())
    perm = bsp.reorder_rcm_host(A.rowptr, A.colidx)
    assert np.array_equal(np.sort(perm), np.arange(9))
    # each component stays contiguous in the new order
    pos = np.empty(9, int)
    pos[perm] = np.arange(9)
    for comp in ({0, 1, 2}, {4, 5, 6, 7, 8}):
        p = sorted(pos[list(comp)])
        assert p[-1] - p[0] == len(comp) - 1


def test_rcm_rejects_bad_input():
    empty = bsp.reorder_rcm_host(np.zeros(1, np.int32), np.zeros(0, np.int32))
    assert empty.size == 0
    with pytest.raises(bsp.BspError):
        bsp.reorder_rcm_host(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32))   # decreasing rowptr
    A = bsp.gen_laplace2d(4, 4)
    with pytest.raises(bsp.BspError):
        bsp.permute_csr_host(A, np.zeros(A.rows, np.int32))                              # not a permutation


@pytest.mark.gpu
def test_device_reorder_matches_host_and_raises_tile_fill(cuda):
    import torch
    A = bsp.gen_stencil27(16, 4, 5)                       # 16,384 rows, dense 4x4 node blocks
    B = _scramble(A, 3)
    rp, ci, va = (torch.from_numpy(a).to(cuda) for a in (B.rowptr, B.colidx, B.values))
    perm = bsp.reorder_rcm(rp, ci)
    assert np.array_equal(perm.cpu().numpy(), bsp.reorder_rcm_host(B.rowptr, B.colidx))
    rp2, ci2, va2 = bsp.permute_csr(rp, ci, va, perm)
    R = bsp.permute_csr_host(B, perm.cpu().numpy())
    assert np.array_equal(rp2.cpu().numpy(), R.rowptr) and np.array_equal(ci2.cpu().numpy(), R.colidx)
    assert np.array_equal(va2.cpu().numpy(), R.values)
    before = bsp.SmatMatrix(rp, ci, va, rows=B.rows, cols=B.cols, dtype="f16")
    after = bsp.SmatMatrix(rp2, ci2, va2, rows=B.rows, cols=B.cols, dtype="f16")
    assert after.fill > 4 * before.fill, (before.fill, after.fill)
    # y = P A P^T (P x) = P (A x): SpMM on the reordered matrix, rows mapped back
    X = torch.rand(B.cols, 128, generator=torch.Generator().manual_seed(1)).half()
    Y0 = before.spmm(X.to(cuda)).cpu().numpy()
    Xp = X[perm.cpu().long()]
    Y1 = after.spmm(Xp.to(cuda)).cpu().numpy()
    assert np.allclose(Y1, Y0[perm.cpu().numpy()], rtol=1e-4, atol=1e-4)
    before.free()
    after.free()
