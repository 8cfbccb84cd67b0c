"""Batched SpMV / 8-RHS SpMM (one persistent launch over many matrices)
against the CPU oracle's FP64 SpMV / SpMM, with the error bound
2*gamma_L*sum|a_ij x_j| (u = 2^-53 for F64, 2^-24 for F32 on inputs already
rounded to F32).  The batched launch, the per-matrix launches, the graph and
the plain launch must agree bit for bit (fixed sum order per output)."""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _small_batch(seed, count=20):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        n = int(rng.integers(50, 3000))
        if i % 3 == 0:
            mats.append(bsp.gen_banded(n, int(rng.integers(3, 28)), seed + i))
        elif i % 3 == 1:
            mats.append(bsp.gen_powerlaw(n, 2.2, n, seed + i))
        else:   # long rows and empty rows
            lens = rng.integers(0, 12, n)
            lens[rng.integers(0, n, 3)] = rng.integers(n // 2, n, 3)
            lens[::7] = 0
            rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
            ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
            mats.append(bsp.HostCSR(n, n, rp, ci, rng.standard_normal(rp[-1])))
    return mats


def _upload(cuda, mats, dtype, nrhs, seed):
    import torch
    tdt = torch.float64 if dtype == "f64" else torch.float32
    rng = np.random.default_rng(seed)
    dev, host = [], []
    for A in mats:
        vals = A.values.astype(np.float32).astype(np.float64) if dtype == "f32" else A.values
        x = rng.uniform(-1, 1, (A.cols, nrhs) if nrhs > 1 else A.cols)
        if dtype == "f32":
            x = x.astype(np.float32).astype(np.float64)
        y = torch.full((A.rows, nrhs) if nrhs > 1 else (A.rows,), float("nan"), dtype=tdt, device=cuda)
        dev.append((torch.from_numpy(A.rowptr).to(cuda), torch.from_numpy(A.colidx).to(cuda),
                    torch.from_numpy(vals).to(tdt).to(cuda), torch.from_numpy(x).to(tdt).to(cuda), y))
        host.append((vals, x))
    return dev, host


def _check(mats, dev, host, dtype, nrhs):
    unit = 2.0 ** -53 if dtype == "f64" else 2.0 ** -24
    for A, (_, _, _, _, y), (vals, x) in zip(mats, dev, host):
        got = y.cpu().numpy().astype(np.float64)
        if nrhs == 1:
            want = pyoracle.spmv_f64(A.rowptr, A.colidx, vals, x)
            tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, vals, x, unit)
        else:
            want, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals, x)
            L = (np.diff(A.rowptr).astype(np.float64) + 1.0)[:, None]
            tol = 2.0 * (L * unit / (1 - L * unit)) * absC + np.finfo(np.float64).tiny
        assert np.all(np.abs(got - want) <= tol)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("nrhs", [1, 8])
def test_batch_matches_oracle_and_separate_launches(cuda, dtype, nrhs):
    import torch
    mats = _small_batch(11 + nrhs)
    dev, host = _upload(cuda, mats, dtype, nrhs, 3)
    P = bsp.BatchPlan(dev, nrhs=nrhs, long_row_nnz=256, seg_nnz=64)
    st = P.stats()
    assert st["long_segments"] > 0 and st["nnz"] == sum(int(A.rowptr[-1]) for A in mats)
    P.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, dtype, nrhs)
    first = [d[4].clone() for d in dev]
    for d in dev:
        d[4].fill_(float("nan"))
    P.run_separate()
    for a, d in zip(first, dev):
        assert torch.equal(a, d[4])
    for _ in range(3):   # counters reset themselves between launches
        P.run()
    for a, d in zip(first, dev):
        assert torch.equal(a, d[4])
    P.close()


def test_batch_graph_and_plain_launch_agree(cuda):
    import torch
    mats = _small_batch(5)
    dev, host = _upload(cuda, mats, "f64", 1, 8)
    P1 = bsp.BatchPlan(dev, long_row_nnz=128, seg_nnz=32, use_graph=True)
    P1.run()
    a = [d[4].clone() for d in dev]
    P2 = bsp.BatchPlan(dev, long_row_nnz=128, seg_nnz=32, use_graph=False)
    P2.run()
    torch.cuda.synchronize()
    for u, d in zip(a, dev):
        assert torch.equal(u, d[4])
    P1.close()
    P2.close()


def test_batch_tuner_choices_and_results(cuda):
    mats = _small_batch(21, count=12)
    dev, host = _upload(cuda, mats, "f64", 1, 9)
    P = bsp.BatchPlan(dev, tune=1)
    lanes = P.lanes()
    assert set(lanes.tolist()) <= {0, 1, 2, 4, 8, 16, 32}
    assert np.array_equal(lanes == 0, P.formats() != 0)     # lanes 0 = stored as SELL-32
    P.run()
    _check(mats, dev, host, "f64", 1)
    P.close()


def test_batch_set_vectors_and_empty_matrix(cuda):
    import torch
    mats = _small_batch(31, count=6)
    mats.append(bsp.HostCSR(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)))
    dev, host = _upload(cuda, mats, "f64", 1, 10)
    P = bsp.BatchPlan(dev)
    A = mats[2]
    x2 = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, A.cols)).to(cuda)
    y2 = torch.empty(A.rows, dtype=torch.float64, device=cuda)
    P.set_vectors(2, x2, y2)
    P.run()
    torch.cuda.synchronize()
    host[2] = (host[2][0], x2.cpu().numpy())
    dev[2] = (*dev[2][:3], x2, y2)
    _check(mats, dev, host, "f64", 1)
    P.close()


def test_batch_rejects_bad_arguments(cuda):
    import torch
    mats = _small_batch(41, count=2)
    dev, _ = _upload(cuda, mats, "f64", 1, 1)
    with pytest.raises(bsp.BspError):
        bsp.BatchPlan(dev, seg_nnz=16)
    with pytest.raises(bsp.BspError):
        bsp.BatchPlan(dev, nrhs=3)
    bad = [(dev[0][0], dev[0][1], dev[0][2].float(), dev[0][3].float(), dev[0][4].float())]
    P = bsp.BatchPlan(bad)   # F32 is fine
    P.close()
    with pytest.raises(ValueError):
        bsp.BatchPlan([(dev[0][0], dev[0][1], dev[0][2].half(), dev[0][3].half(), dev[0][4].half())])
    _ = torch


def _sell_batch(seed):
    """Banded matrices (even rows: SELL-32), a rectangular banded block, a
    matrix whose columns reach 40,000 from their rows (int16 offsets do not
    fit: stays CSR), power-law rows (uneven: CSR), and a banded matrix with
    every 5th row empty (padding over 1/8: CSR)."""
    rng = np.random.default_rng(seed)
    mats = [bsp.gen_banded(int(rng.integers(100, 5000)), int(w), seed + i) for i, w in enumerate((3, 9, 15, 27))]
    B = bsp.gen_banded(3000, 11, seed + 7)
    keep = B.rowptr[2000]
    mats.append(bsp.HostCSR(2000, 3000, B.rowptr[:2001].copy(), B.colidx[:keep].copy(), B.values[:keep].copy()))
    n = 50000
    rp = np.arange(0, 2 * n + 1, 2, dtype=np.int32)
    ci = np.stack([np.arange(n), (np.arange(n) + 40000) % n], 1)
    ci.sort(axis=1)
    mats.append(bsp.HostCSR(n, n, rp, ci.reshape(-1).astype(np.int32), rng.standard_normal(2 * n)))
    mats.append(bsp.gen_powerlaw(8000, 2.2, 8000, seed + 9))
    E = bsp.gen_banded(1000, 9, seed + 11)
    lens = np.diff(E.rowptr)
    lens[::5] = 0
    keepmask = np.repeat(lens > 0, np.diff(E.rowptr))
    erp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    mats.append(bsp.HostCSR(1000, 1000, erp, E.colidx[keepmask].copy(), E.values[keepmask].copy()))
    return mats


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("nrhs", [1, 8])
def test_batch_sell_format_choice_and_results(cuda, dtype, nrhs):
    import torch
    mats = _sell_batch(70 + nrhs)
    dev, host = _upload(cuda, mats, dtype, nrhs, 12)
    P = bsp.BatchPlan(dev, nrhs=nrhs, long_row_nnz=1024, seg_nnz=256)
    fm = P.formats()
    assert fm.tolist() == [1, 1, 1, 1, 1, 0, 0, 0]
    assert P.lanes()[:5].tolist() == [0] * 5 and P.lanes()[5:].min() >= 1
    P.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, dtype, nrhs)
    first = [d[4].clone() for d in dev]
    for d in dev:
        d[4].fill_(float("nan"))
    P.run_separate()
    for a, d in zip(first, dev):
        assert torch.equal(a, d[4])
    Q = bsp.BatchPlan(dev, nrhs=nrhs, sell=False)
    assert not Q.formats().any()
    Q.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, dtype, nrhs)
    T = bsp.BatchPlan(dev, nrhs=nrhs, tune=1, long_row_nnz=1024, seg_nnz=256)
    assert np.array_equal(T.formats(), fm)      # SELL by the eligibility rule, lanes timed for the rest
    T.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, dtype, nrhs)
    for X in (P, Q, T):
        X.close()


@pytest.mark.parametrize("nrhs", [1, 8])
def test_batch_wide_sell_form(cuda, nrhs):
    """The opt-in wide SELL-32 form: the power-law matrix and the banded one
    with empty rows (both uneven in row order) are stored as length-sorted
    SELL-32 with their longest rows as whole-warp segments; results within
    the bound and identical between the batched and the separate launches."""
    import torch
    mats = _sell_batch(90 + nrhs)
    dev, host = _upload(cuda, mats, "f64", nrhs, 13)
    P = bsp.BatchPlan(dev, nrhs=nrhs, long_row_nnz=1024, seg_nnz=256, sell_wide=True)
    assert P.formats().tolist() == [1, 1, 1, 1, 1, 0, 2, 2]
    P.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, "f64", nrhs)
    first = [d[4].clone() for d in dev]
    P.run_separate()
    for a, d in zip(first, dev):
        assert torch.equal(a, d[4])
    P.close()


def _even_rows(rows, cols, per_row, span, seed):
    """Every row `per_row` distinct columns within `span` of min(row, cols - 1):
    even rows, so the batch stores the matrix as SELL-32."""
    rng = np.random.default_rng(seed)
    ci = []
    for r in range(rows):
        c0 = min(r, cols - 1)
        lo, hi = max(0, c0 - span), min(cols, c0 + span + 1)
        ci.append(np.sort(rng.choice(np.arange(lo, hi), per_row, replace=False)))
    rp = np.arange(rows + 1, dtype=np.int32) * per_row
    return bsp.HostCSR(rows, cols, rp, np.concatenate(ci).astype(np.int32), rng.standard_normal(rows * per_row))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_batch_sell_slices_with_and_without_x_window(cuda, dtype):
    """8 right-hand sides on SELL-32 matrices: slices whose columns lie within
    64 rows gather x from a shared-memory window (FP64), the others from
    global memory; a rectangular matrix clips the window at its last column,
    and a partial last slice has fewer than 32 rows.  Results against the
    oracle, and the batched launch against the per-matrix launches."""
    import torch
    mats = [bsp.gen_banded(1000, 9, 1),                    # every slice windowed, last slice partial
            _even_rows(777, 777, 8, 3000, 2),             # no slice windowed
            _even_rows(1000, 700, 6, 12, 3),              # rectangular: window clipped at 700 columns
            _even_rows(640, 640, 4, 40, 4)]               # spans just above and below the window
    half = _even_rows(512, 512, 5, 6, 5)                  # banded rows, then scattered rows in one matrix
    wide = _even_rows(512, 512, 5, 400, 6)
    rp = np.concatenate([half.rowptr[:257], wide.rowptr[257:] - wide.rowptr[256] + half.rowptr[256]]).astype(np.int32)
    ci = np.concatenate([half.colidx[:half.rowptr[256]], wide.colidx[wide.rowptr[256]:]]).astype(np.int32)
    mats.append(bsp.HostCSR(512, 512, rp, ci, np.random.default_rng(7).standard_normal(ci.size)))
    dev, host = _upload(cuda, mats, dtype, 8, 12)
    P = bsp.BatchPlan(dev, nrhs=8)
    assert np.all(P.formats() == 1), P.formats()
    P.run()
    torch.cuda.synchronize()
    _check(mats, dev, host, dtype, 8)
    first = [d[4].clone() for d in dev]
    for d in dev:
        d[4].fill_(float("nan"))
    P.run_separate()
    for a, d in zip(first, dev):
        assert torch.equal(a, d[4])
    P.close()
