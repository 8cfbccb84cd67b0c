"""Reverse Cuthill-McKee reordering and symmetric permutation: valid
permutations, bandwidth as small as scipy's RCM, P A P^T exact, components
and edge cases on the host; on the GPU the device forms agree with the host
forms and reordering a scrambled stencil raises the SMaT 16x16 tile fill.
Row-similarity order: row-shuffled tile matrices regrouped to the original
tile count, noisy groups, P A exact, group sizes, empty rows, bad input, and
the SpMM engine choice that uses it; on the GPU the device forms agree and
the reordered SMaT product is the shuffled one with rows permuted."""
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


# --- row-similarity order -------------------------------------------------

def _grouped(groups, blocks, nblocks, seed, keep=1.0, G=16, BC=16):
    """groups x G rows; the rows of a group draw from the same `blocks`
    column blocks (each block kept with probability `keep`, at least one);
    rows then shuffled.  Returns (scrambled, original) HostCSR."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for g in range(groups):
        bset = np.sort(rng.choice(nblocks, blocks, replace=False))
        for r in range(G):
            kept = bset[rng.random(blocks) < keep]
            if kept.size == 0:
                kept = bset[:1]
            c = (kept[:, None] * BC + np.arange(BC)[None, :]).ravel()
            rows.append(np.full(c.size, g * G + r))
            cols.append(c)
            vals.append(rng.uniform(-1, 1, c.size))
    M = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(groups * G, nblocks * BC))
    M.sort_indices()
    p = np.random.default_rng(seed + 1).permutation(M.shape[0])
    S = M[p].tocsr()
    S.sort_indices()
    mk = lambda X: bsp.HostCSR(X.shape[0], X.shape[1], X.indptr.astype(np.int32), X.indices.astype(np.int32),
                               X.data.copy())
    return mk(S), mk(M)


def _tiles(A, G=16, BC=16):
    r = np.repeat(np.arange(A.rows), np.diff(A.rowptr)) // G
    return np.unique(r.astype(np.int64) * (A.cols // BC + 1) + A.colidx // BC).size


def test_similarity_regroups_scrambled_tiles_exactly():
    S, M = _grouped(256, 6, 1024, 11)
    assert _tiles(S) > 10 * _tiles(M)
    perm = bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols)
    assert np.array_equal(np.sort(perm), np.arange(S.rows))
    R = bsp.permute_rows_csr_host(S, perm)
    assert _tiles(R) == _tiles(M) == 256 * 6
    assert np.array_equal(perm, bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols))   # deterministic


def test_similarity_groups_noisy_rows():
    S, M = _grouped(300, 8, 2048, 12, keep=0.7)
    R = bsp.permute_rows_csr_host(S, bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols))
    assert _tiles(R) <= 1.25 * _tiles(M) and _tiles(S) > 5 * _tiles(R), (_tiles(S), _tiles(R), _tiles(M))


def test_permute_rows_is_row_indexing():
    S, _ = _grouped(20, 3, 64, 13)
    perm = np.random.default_rng(3).permutation(S.rows).astype(np.int32)
    R = bsp.permute_rows_csr_host(S, perm)
    ref = _scipy(S)[perm].tocsr()
    assert np.array_equal(R.rowptr, ref.indptr) and np.array_equal(R.colidx, ref.indices)
    assert np.array_equal(R.values, ref.data) and (R.rows, R.cols) == (S.rows, S.cols)


def test_similarity_group_size_empty_rows_and_bad_input():
    S, M = _grouped(40, 4, 100, 14, G=8, BC=8)
    perm = bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols, group_rows=8, block_cols=8)
    assert _tiles(bsp.permute_rows_csr_host(S, perm), 8, 8) == _tiles(M, 8, 8)
    # empty rows (3 of them) are placed last, in row order
    rp = np.array([0, 2, 2, 3, 3, 5, 5], np.int32)
    ci = np.array([0, 17, 1, 16, 18], np.int32)
    perm = bsp.reorder_similarity_host(rp, ci, 32, group_rows=2)
    assert np.array_equal(np.sort(perm), np.arange(6)) and list(perm[3:]) == [1, 3, 5]
    assert bsp.reorder_similarity_host(np.zeros(1, np.int32), np.zeros(0, np.int32), 0).size == 0
    for bad in (dict(group_rows=0), dict(block_cols=0)):
        with pytest.raises(bsp.BspError):
            bsp.reorder_similarity_host(rp, ci, 32, **bad)
    with pytest.raises(bsp.BspError):
        bsp.reorder_similarity_host(rp, ci, 18)                                          # column 18 >= cols
    with pytest.raises(bsp.BspError):
        bsp.permute_rows_csr_host(S, np.zeros(S.rows, np.int32))                         # not a permutation


def _argmin_engine(d):
    est = {"csr": d["est_seconds_csr"]}
    for e in ("smat", "gtile"):
        for o in ("given", "reordered"):
            if d[f"est_seconds_{e}_{o}"] >= 0:
                est[f"{e}_{o}"] = d[f"est_seconds_{e}_{o}"]
    return min(est, key=lambda k: (est[k], k))


def _chunks(A, perm=None):
    """Gathered-tile chunks: ceil(distinct columns / 16) per 16-row group."""
    order = np.arange(A.rows) if perm is None else perm
    total = 0
    for g in range(0, A.rows, 16):
        cols = [A.colidx[A.rowptr[r]:A.rowptr[r + 1]] for r in order[g:g + 16]]
        total += (np.unique(np.concatenate(cols)).size + 15) // 16
    return total


def _permute_columns(A, seed):
    perm = np.random.default_rng(seed).permutation(A.cols).astype(np.int32)
    rows = np.repeat(np.arange(A.rows, dtype=np.int32), np.diff(A.rowptr))
    nc = perm[A.colidx]
    o = np.lexsort((nc, rows))
    return bsp.HostCSR(A.rows, A.cols, A.rowptr, np.ascontiguousarray(nc[o]), np.ascontiguousarray(A.values[o]))


def test_spmm_choice_uses_the_similarity_order():
    S, M = _grouped(256, 6, 1024, 11)
    d, perm = bsp.choose_spmm_host(S, 128)
    assert (d["engine"], d["reorder"], d["smat_path"]) == ("smat", True, "tcgen05")
    assert np.array_equal(perm, bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols))
    assert d["tiles_given"] == _tiles(S) and d["tiles_reordered"] == _tiles(M) == 256 * 6
    assert _argmin_engine(d) == "smat_reordered"
    d, _ = bsp.choose_spmm_host(M, 128)                        # already grouped: no reordering needed
    assert (d["engine"], d["reorder"]) == ("smat", False) and _argmin_engine(d) == "smat_given"


def test_spmm_choice_scattered_rows_and_n():
    G = bsp.gen_graph(1 << 16, 1.8, 8, 7)                      # power-law graph: few nonzeros per tile
    d, _ = bsp.choose_spmm_host(G, 128)
    assert d["engine"] == "csr" and _argmin_engine(d) == "csr"
    S, _ = _grouped(64, 4, 256, 16)
    d, perm = bsp.choose_spmm_host(S, 96, reorder=False)        # N % 128 != 0: tcgen05 in 64-column slabs
    assert perm is None and d["tiles_reordered"] == -1 and d["est_seconds_smat_reordered"] == -1.0
    assert d["smat_path"] == "tcgen05" and d["engine"] == {"csr": "csr", "smat_given": "smat"}[_argmin_engine(d)]
    d, _ = bsp.choose_spmm_host(S, 100)                         # SMaT needs N % 32 == 0
    assert d["engine"] == "csr" and d["est_seconds_smat_given"] == -1.0
    with pytest.raises(bsp.BspError):
        bsp.choose_spmm_host(S, 0)


def test_spmm_choice_picks_gathered_tiles_for_shared_scattered_columns():
    """A stencil with its columns permuted: 16x16 tiles are almost empty but
    the rows of a 16-row group share their columns, so the gathered-tile
    chunks are half full and that engine is estimated fastest."""
    P = _permute_columns(bsp.gen_stencil27(8, 4, 3), 5)
    d, perm = bsp.choose_spmm_host(P, 128)
    assert d["chunks_given"] == _chunks(P) and d["chunks_reordered"] == _chunks(P, perm)
    assert d["engine"] == "gtile" and d["engine"] == _argmin_engine(d).split("_")[0]
    assert P.nnz / (16 * 16 * d["chunks_given"]) > 0.4 and P.nnz / (256 * d["tiles_given"]) < 0.1
    d, _ = bsp.choose_spmm_host(P, 100, reorder=False)          # the gathered tiles need N % 8 == 0
    assert d["est_seconds_gtile_given"] == -1.0 and d["chunks_reordered"] == -1 and d["engine"] == "csr"
    d, _ = bsp.choose_spmm_host(P, 104, reorder=False)
    assert d["engine"] == "gtile" and d["reorder"] is False


@pytest.mark.gpu
def test_device_similarity_matches_host_and_densifies_tiles(cuda):
    import torch
    S, M = _grouped(2048, 6, 4096, 15)                   # 32,768 rows, scrambled dense 16x16 tiles
    rp, ci, va = (torch.from_numpy(a).to(cuda) for a in (S.rowptr, S.colidx, S.values))
    perm = bsp.reorder_similarity(rp, ci, S.cols)
    assert np.array_equal(perm.cpu().numpy(), bsp.reorder_similarity_host(S.rowptr, S.colidx, S.cols))
    rp2, ci2, va2 = bsp.permute_rows_csr(rp, ci, va, perm)
    R = bsp.permute_rows_csr_host(S, perm.cpu().numpy())
    assert np.array_equal(rp2.cpu().numpy(), R.rowptr) and np.array_equal(ci2.cpu().numpy(), R.colidx)
    assert np.array_equal(va2.cpu().numpy(), R.values)
    before = bsp.SmatMatrix(rp, ci, va, rows=S.rows, cols=S.cols, dtype="f16")
    after = bsp.SmatMatrix(rp2, ci2, va2, rows=S.rows, cols=S.cols, dtype="f16")
    assert after.fill == 1.0 and after.fill > 10 * before.fill, (before.fill, after.fill)
    # (P A) X = P (A X): row i of the reordered product is row perm[i]
    X = (torch.rand(S.cols, 128, generator=torch.Generator().manual_seed(2)) * 2 - 1).half().to(cuda)
    Y0 = before.spmm(X).cpu().numpy()
    Y1 = after.spmm(X).cpu().numpy()
    assert np.allclose(Y1, Y0[perm.cpu().numpy()], rtol=1e-4, atol=1e-4)
    before.free()
    after.free()
