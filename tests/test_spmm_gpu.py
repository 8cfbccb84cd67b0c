"""SpMM on the GPU (C = alpha*A*B + beta*C, FP32 accumulation): the CSR path,
the row-split CSR path for power-law rows, and the 16x16-tile tensor-core
(SMaT) path, each against the CPU oracle's FP64 SpMM of the same quantized
inputs.  Products of two F16 (or two BF16) numbers are exact in FP32, so the
only error is FP32 accumulation: |C - C_fp64| <= 2*gamma_L*(|A||B|) with
gamma_L = L*u/(1-L*u), u = 2^-24, L = row length + 2 (the tolerance below)."""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu

_NP = {"f16": np.float16, "bf16": None, "f32": np.float32}


def _torch_dtype(name):
    import torch
    return {"f16": torch.float16, "bf16": torch.bfloat16, "f32": torch.float32}[name]


def _quantize(a: np.ndarray, name: str):
    """Rounds FP64 data to `name` on the host; returns (torch CPU tensor of that
    dtype, FP64 copy of the rounded values)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(_torch_dtype(name))
    return t, t.to(torch.float64).numpy()


def _tol(A, absC, alpha=1.0, Cin=None, beta=0.0):
    L = (np.diff(A.rowptr).astype(np.float64) + 2.0)[:, None]
    u = 2.0 ** -24
    g = L * u / (1.0 - L * u)
    t = 2.0 * g * abs(alpha) * absC + 1e-30
    if Cin is not None:
        t = t + 4.0 * u * (abs(alpha) * absC + abs(beta) * np.abs(Cin))
    return t


def _case(A, N, name, seed):
    rng = np.random.default_rng(seed)
    vals_t, vals64 = _quantize(A.values, name)
    B_t, B64 = _quantize(rng.uniform(-1, 1, (A.cols, N)), name)
    return vals_t, vals64, B_t, B64


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


@pytest.mark.parametrize("name", ["f16", "bf16", "f32"])
@pytest.mark.parametrize("N", [32, 40, 128, 256])
def test_spmm_csr_matches_fp64(cuda, name, N):
    A = bsp.gen_powerlaw(3001, 1.6, 700, 9)
    vals_t, vals64, B_t, B64 = _case(A, N, name, N)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    C = bsp.spmm_csr(rp, ci, vals_t.to(cuda), B_t.to(cuda)).cpu().numpy().astype(np.float64)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    assert np.all(np.abs(C - Cref) <= _tol(A, absC))


@pytest.mark.parametrize("name", ["f16", "bf16"])
def test_spmm_csr_alpha_beta(cuda, name):
    import torch
    A = bsp.gen_powerlaw(1500, 1.8, 300, 3)
    N = 64
    vals_t, vals64, B_t, B64 = _case(A, N, name, 5)
    Cin = np.random.default_rng(1).uniform(-1, 1, (A.rows, N)).astype(np.float32)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    Cd = torch.from_numpy(Cin.copy()).to(cuda)
    bsp.spmm_csr(rp, ci, vals_t.to(cuda), B_t.to(cuda), Cd, alpha=0.5, beta=-1.5)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    want = 0.5 * Cref - 1.5 * Cin.astype(np.float64)
    got = Cd.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(got - want) <= _tol(A, absC, 0.5, Cin, -1.5))


@pytest.mark.parametrize("chunk", [32, 64, 256])
@pytest.mark.parametrize("N", [32, 128])
def test_spmm_planned_matches_fp64_and_is_deterministic(cuda, chunk, N):
    A = bsp.gen_powerlaw(4000, 1.4, 3000, 17)   # rows up to 3000 long
    assert np.diff(A.rowptr).max() > 4 * chunk
    vals_t, vals64, B_t, B64 = _case(A, N, "f16", chunk + N)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    vd, Bd = vals_t.to(cuda), B_t.to(cuda)
    P = bsp.SpmmPlan(rp, ci, vd, cols=A.cols, chunk=chunk)
    lens = np.diff(A.rowptr)
    assert P.nsplit == int(np.sum(lens > chunk))
    assert P.nchunks == int(np.sum(np.maximum(1, (lens + chunk - 1) // chunk)))
    C1 = P.spmm(Bd).cpu().numpy()
    C2 = P.spmm(Bd).cpu().numpy()
    assert np.array_equal(C1, C2)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    assert np.all(np.abs(C1.astype(np.float64) - Cref) <= _tol(A, absC))
    P.free()


@pytest.mark.parametrize("name", ["f16", "f32"])
def test_spmm_csr_long_row_goes_through_a_temporary_plan(cuda, name):
    """A row of 20,000 nonzeros among rows of ~4: the plan-free call splits it
    (a temporary row-split plan with 256-nonzero chunks), giving exactly the
    planned result, within the FP32 accumulation bound of the FP64 oracle."""
    import torch
    rng = np.random.default_rng(8)
    n = 30000
    lens = rng.integers(0, 8, n)
    lens[123] = 20000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in lens]).astype(np.int32)
    A = bsp.HostCSR(n, n, rp, ci, rng.uniform(-1, 1, int(rp[-1])))
    N = 64
    vals_t, vals64, B_t, B64 = _case(A, N, name, 5)
    ref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    rpd, cid = _dev(cuda, A.rowptr, A.colidx)
    vd, Bd = vals_t.to(cuda), B_t.to(cuda)
    C1 = bsp.spmm_csr(rpd, cid, vd, Bd)
    P = bsp.SpmmPlan(rpd, cid, vd, cols=A.cols, chunk=256)
    C2 = P.spmm(Bd)
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)
    assert np.all(np.abs(C1.cpu().numpy().astype(np.float64) - ref) <= _tol(A, absC))
    P.free()


def test_spmm_planned_empty_rows_and_beta(cuda):
    import torch
    # every third row empty
    rng = np.random.default_rng(2)
    rows, cols = 900, 700
    lens = rng.integers(0, 600, rows)
    lens[::3] = 0
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    colidx = np.concatenate([np.sort(rng.choice(cols, l, replace=False)) for l in lens]).astype(np.int32)
    A = bsp.HostCSR(rows, cols, rowptr, colidx, rng.uniform(-1, 1, rowptr[-1]))
    N = 32
    vals_t, vals64, B_t, B64 = _case(A, N, "bf16", 8)
    Cin = rng.uniform(-1, 1, (rows, N)).astype(np.float32)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    P = bsp.SpmmPlan(rp, ci, vals_t.to(cuda), cols=cols, chunk=128)
    Cd = torch.from_numpy(Cin.copy()).to(cuda)
    P.spmm(B_t.to(cuda), Cd, alpha=2.0, beta=0.25)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    want = 2.0 * Cref + 0.25 * Cin.astype(np.float64)
    got = Cd.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(got - want) <= _tol(A, absC, 2.0, Cin, 0.25))
    assert np.array_equal(got[::3], (0.25 * Cin[::3]).astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("name", ["f16", "bf16"])
@pytest.mark.parametrize("N", [32, 64, 256])
@pytest.mark.parametrize("kind", ["dense_tiles", "ragged"])
def test_smat_block_spmm_matches_fp64(cuda, name, N, kind):
    if kind == "dense_tiles":
        A = bsp.gen_random_bsr(96, 16, 6, 1.0, 1.0, 4)
    else:   # partially filled tiles, rows/cols not multiples of 16
        A = bsp.gen_powerlaw(1003, 1.7, 400, 12)
    vals_t, vals64, B_t, B64 = _case(A, N, name, N + 1)
    rp, ci, v64 = _dev(cuda, A.rowptr, A.colidx, vals64)
    M = bsp.SmatMatrix(rp, ci, v64, rows=A.rows, cols=A.cols, dtype=name)
    if kind == "dense_tiles":
        assert M.fill == 1.0
    C1 = M.spmm(B_t.to(cuda))
    M.check()
    C1 = C1.cpu().numpy()
    C2 = M.spmm(B_t.to(cuda)).cpu().numpy()
    assert np.array_equal(C1, C2)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    # the tile MMA sums 16 products per step in an unspecified order: bound
    # with the full tile row length instead of the CSR row length
    tiles_per_row = (A.cols + 15) // 16
    L = np.full((A.rows, 1), 16.0 * tiles_per_row + 2.0)
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1 - L * u)) * absC + 1e-30
    assert np.all(np.abs(C1.astype(np.float64) - Cref) <= tol)
    M.free()


def test_smat_alpha_beta_and_argument_errors(cuda):
    import torch
    A = bsp.gen_random_bsr(40, 16, 4, 0.5, 1.0, 6)
    N = 32
    vals_t, vals64, B_t, B64 = _case(A, N, "f16", 3)
    rp, ci, v64 = _dev(cuda, A.rowptr, A.colidx, vals64)
    M = bsp.SmatMatrix(rp, ci, v64, rows=A.rows, cols=A.cols, dtype="f16")
    Cin = np.random.default_rng(4).uniform(-1, 1, (A.rows, N)).astype(np.float32)
    Cd = torch.from_numpy(Cin.copy()).to(cuda)
    M.spmm(B_t.to(cuda), Cd, alpha=-1.0, beta=0.5)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    want = -Cref + 0.5 * Cin.astype(np.float64)
    L = np.full((A.rows, 1), 16.0 * ((A.cols + 15) // 16) + 2.0)
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1 - L * u)) * absC + 4 * u * (absC + 0.5 * np.abs(Cin)) + 1e-30
    assert np.all(np.abs(Cd.cpu().numpy().astype(np.float64) - want) <= tol)
    with pytest.raises(bsp.BspError):
        M.spmm(torch.zeros(A.cols, 40, dtype=torch.float16, device=cuda))   # N not a multiple of 32
    with pytest.raises(ValueError):
        bsp.spmm_csr(rp, ci, vals_t.to(cuda), B_t.to(cuda).to(torch.bfloat16))
    M.free()


@pytest.mark.parametrize("name", ["f16", "bf16"])
@pytest.mark.parametrize("N", [32, 64, 96, 128, 256])
@pytest.mark.parametrize("kind", ["dense_tiles", "ragged"])
def test_smat_tcgen05_and_mma_sync_paths(cuda, name, N, kind):
    """The tcgen05 path (TMEM accumulator, TMA-staged B) at both slab widths
    (64 and 128 C columns per CTA; columns past N zero-filled by TMA and not
    stored), its persistent warp-specialised form (empty block rows and
    more block rows than resident CTAs included) and the mma.sync path
    against the FP64 oracle; all deterministic across calls."""
    import torch
    A = bsp.gen_random_bsr(96, 16, 6, 1.0, 1.0, 4) if kind == "dense_tiles" else bsp.gen_powerlaw(1003, 1.7, 400, 12)
    vals_t, vals64, B_t, B64 = _case(A, N, name, N + 7)
    rp, ci, v64 = _dev(cuda, A.rowptr, A.colidx, vals64)
    M = bsp.SmatMatrix(rp, ci, v64, rows=A.rows, cols=A.cols, dtype=name)
    Bd = B_t.to(cuda)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    L = np.full((A.rows, 1), 16.0 * ((A.cols + 15) // 16) + 2.0)
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1 - L * u)) * absC + 1e-30
    for path in ("tcgen05", "tcgen05_w64", "tcgen05_w128", "tcgen05_persistent", "tcgen05_persistent_w64", "mma_sync"):
        C1 = M.spmm(Bd, path=path).cpu().numpy()
        C2 = M.spmm(Bd, path=path).cpu().numpy()
        M.check()
        assert np.array_equal(C1, C2), path
        assert np.all(np.abs(C1.astype(np.float64) - Cref) <= tol), path
    Cin = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, (A.rows, N)).astype(np.float32)).to(cuda)
    Cb = M.spmm(Bd, Cin.clone(), alpha=0.5, beta=2.0, path="tcgen05").cpu().numpy().astype(np.float64)
    want = 0.5 * Cref + 2.0 * Cin.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(Cb - want) <= tol + 4 * u * (0.5 * absC + 2.0 * np.abs(Cin.cpu().numpy())))
    with pytest.raises(bsp.BspError):
        M.spmm(torch.zeros(A.cols, 48, dtype=Bd.dtype, device=cuda), path="tcgen05")   # N % 32 != 0
    M.free()


@pytest.mark.parametrize("name", ["f16", "bf16", "f32"])
@pytest.mark.parametrize("N,slab", [(32, 0), (64, 16), (128, 32), (128, 64), (256, 32), (40, 8), (256, 256)])
def test_spmm_slab_engine_matches_fp64(cuda, name, N, slab):
    """The slab engine (column slabs, length-sorted short rows one per lane
    group, long-row chunks a warp each): every slab width against the FP64
    oracle within the FP32 accumulation bound, with long rows (split into
    chunks), empty rows, and alpha/beta; repeat calls give the same bits."""
    import torch
    if name == "f32" and slab > 128:
        pytest.skip("F32 slabs are at most 32 lanes x 4 columns")
    if name != "f32" and (N % 8 or (slab and slab % 8)):
        pytest.skip("16-bit slabs are multiples of 8 columns")
    rng = np.random.default_rng(N + slab)
    n = 6000
    lens = rng.integers(0, 40, n)
    lens[rng.integers(0, n, 5)] = rng.integers(300, 3000, 5)   # split into 256-nonzero chunks
    lens[::11] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    A = bsp.HostCSR(n, n, rp, ci, rng.uniform(-1, 1, rp[-1]))
    vals_t, vals64, B_t, B64 = _case(A, N, name, 7)
    Cin = rng.uniform(-1, 1, (n, N)).astype(np.float32)
    rpd, cid = _dev(cuda, A.rowptr, A.colidx)
    P = bsp.SpmmPlan(rpd, cid, vals_t.to(cuda), cols=A.cols, chunk=256)
    assert P.nsplit == int(np.sum(lens > 256))
    Bd = B_t.to(cuda)
    C1 = P.spmm(Bd, engine="slab", slab_cols=slab)
    assert torch.equal(C1, P.spmm(Bd, engine="slab", slab_cols=slab))
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    assert np.all(np.abs(C1.cpu().numpy().astype(np.float64) - Cref) <= _tol(A, absC))
    Cd = torch.from_numpy(Cin.copy()).to(cuda)
    P.spmm(Bd, Cd, alpha=0.5, beta=-1.5, engine="slab", slab_cols=slab)
    want = 0.5 * Cref - 1.5 * Cin.astype(np.float64)
    assert np.all(np.abs(Cd.cpu().numpy().astype(np.float64) - want) <= _tol(A, absC, 0.5, Cin, -1.5))
    # the L2 cache policies change where lines stay, not the sums
    for hints in (0, 2, 1):
        P.slab_l2_hints = hints
        assert torch.equal(C1, P.spmm(Bd, engine="slab", slab_cols=slab))
    P.free()


def test_spmm_plan_ranges_match_row_pointers(cuda):
    """The plan's per-slot and per-short-row nonzero ranges agree with the
    row pointers: long-row chunks tile each split row in order, and the
    short-row list is sorted longest first with each row's own range."""
    rng = np.random.default_rng(3)
    n = 3000
    lens = rng.integers(0, 30, n)
    lens[[5, 700, 2999]] = [1000, 257, 2900]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32)
    import torch
    rpd, cid = _dev(cuda, rp, ci)
    v = torch.ones(int(rp[-1]), dtype=torch.float16, device=cuda)
    P = bsp.SpmmPlan(rpd, cid, v, cols=n, chunk=256)
    d = P._d
    from benchsp_b200.api import _d2h
    long_se = _d2h(d.long_se, 2 * d.nparts, np.int32).reshape(-1, 2)
    short_se = _d2h(d.short_se, 2 * d.nshort, np.int32).reshape(-1, 2)
    short_rows = _d2h(d.short_rows, d.nshort, np.int32)
    split = np.flatnonzero(lens > 256)
    want_long = [(rp[r] + k * 256, min(rp[r] + (k + 1) * 256, rp[r + 1]))
                 for r in split for k in range((lens[r] + 255) // 256)]
    assert sorted(map(tuple, long_se.tolist())) == sorted(want_long)
    assert np.array_equal(short_se[:, 0], rp[short_rows]) and np.array_equal(short_se[:, 1], rp[short_rows + 1])
    ln = lens[short_rows]
    assert np.all(ln[:-1] >= ln[1:]) and set(short_rows.tolist()) == set(np.flatnonzero(lens <= 256).tolist())
    P.free()


def test_spmm_slab_engine_rejects_bad_widths(cuda):
    import torch
    A = bsp.gen_powerlaw(500, 1.8, 100, 3)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    v = torch.from_numpy(A.values).to(torch.float16).to(cuda)
    B = torch.zeros(A.cols, 64, dtype=torch.float16, device=cuda)
    P = bsp.SpmmPlan(rp, ci, v, cols=A.cols)
    for bad in (24, 48, 512):   # not a power of two times 8, or wider than N
        with pytest.raises(bsp.BspError):
            P.spmm(B, engine="slab", slab_cols=bad)
    P.free()


@pytest.mark.parametrize("N", [64, 128, 256])
def test_smat_tcgen05_persistent_many_block_rows(cuda, N):
    """Persistent tcgen05 kernel on far more block rows than resident CTAs
    (each CTA walks many block rows, alternating its two TMEM accumulators),
    with every 7th block row empty: the same bits as the one-CTA-per-block-row
    kernel (same MMAs in the same order) and within the FP32 bound."""
    import torch
    A = bsp.gen_random_bsr(3000, 16, 4, 0.5, 1.0, 21)
    keep = (np.arange(A.rows) // 16) % 7 != 0
    lens = np.where(keep, np.diff(A.rowptr), 0)
    mask = np.repeat(keep, np.diff(A.rowptr))
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    A = bsp.HostCSR(A.rows, A.cols, rp, A.colidx[mask].copy(), A.values[mask].copy())
    vals_t, vals64, B_t, B64 = _case(A, N, "f16", 31)
    rpd, cid, v64 = _dev(cuda, A.rowptr, A.colidx, vals64)
    M = bsp.SmatMatrix(rpd, cid, v64, rows=A.rows, cols=A.cols, dtype="f16")
    Bd = B_t.to(cuda)
    Cin = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, (A.rows, N)).astype(np.float32)).to(cuda)
    ref_path = "tcgen05_w128" if N >= 128 else "tcgen05_w64"
    C0 = M.spmm(Bd, Cin.clone(), alpha=1.5, beta=-0.5, path=ref_path)
    for _ in range(2):
        C1 = M.spmm(Bd, Cin.clone(), alpha=1.5, beta=-0.5, path="tcgen05_persistent")
        M.check()
        assert torch.equal(C0, C1)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    want = 1.5 * Cref - 0.5 * Cin.cpu().numpy().astype(np.float64)
    L = np.full((A.rows, 1), 16.0 * ((A.cols + 15) // 16) + 2.0)
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1 - L * u)) * 1.5 * absC + 4 * u * (1.5 * absC + 0.5 * np.abs(Cin.cpu().numpy())) + 1e-30
    assert np.all(np.abs(C1.cpu().numpy().astype(np.float64) - want) <= tol)
    M.free()


@pytest.mark.parametrize("name", ["f16", "bf16"])
@pytest.mark.parametrize("N", [32, 64, 128, 256])
def test_gtile_spmm_matches_fp64(cuda, name, N):
    """Gathered-tile tensor-core SpMM on a power-law graph (rows up to
    thousands of nonzeros, so some 16-row groups span several 64-chunk
    pieces summed through the workspace): each group's chunk columns are its
    distinct columns in ascending order, the product is within the FP32
    bound of the FP64 oracle (L = 16 x the group's chunks + pieces + 2 terms
    per output) and repeat calls give the same bits; alpha and beta."""
    import torch
    A = bsp.gen_graph(12000, 1.6, 16, 5)     # 16 groups of more than 1024 nonzeros
    vals_t, vals64, B_t, B64 = _case(A, N, name, N + 3)
    Aq = bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, vals64)
    G = bsp.GatherTileMatrix(Aq, dtype=name)
    assert G.nsplit > 0 and G.ngroups == (A.rows + 15) // 16
    cpg = G.chunks_per_group()
    cols = bsp.api._d2h(G.chunk_cols, G.nchunks * 16, np.int32).reshape(-1, 16)
    starts = np.concatenate([[0], np.cumsum(cpg)])
    for g in (0, 7, G.ngroups - 1, int(np.argmax(cpg))):
        u = np.unique(A.colidx[A.rowptr[16 * g]:A.rowptr[min(A.rows, 16 * g + 16)]])
        got = cols[starts[g]:starts[g + 1]].reshape(-1)
        assert np.array_equal(got[:u.size], u) and not got[u.size:].any()
    Bd = B_t.to(cuda)
    Cin = torch.from_numpy(np.random.default_rng(N).uniform(-1, 1, (A.rows, N)).astype(np.float32)).to(cuda)
    C1 = G.spmm(Bd, Cin.clone(), alpha=0.75, beta=-2.0)
    C2 = G.spmm(Bd, Cin.clone(), alpha=0.75, beta=-2.0)
    G.check()
    assert torch.equal(C1, C2)
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    want = 0.75 * Cref - 2.0 * Cin.cpu().numpy().astype(np.float64)
    L = (16.0 * np.repeat(cpg, 16)[:A.rows] + 2.0 + 64)[:, None]
    u = 2.0 ** -24
    tol = 2.0 * (L * u / (1 - L * u)) * 0.75 * absC + 4 * u * (0.75 * absC + 2.0 * np.abs(Cin.cpu().numpy())) + 1e-30
    assert np.all(np.abs(C1.cpu().numpy().astype(np.float64) - want) <= tol)
    G.free()


@pytest.mark.parametrize("N", [24, 64, 136])
def test_gtile_column_permuted_stencil(cuda, N):
    """Gathered tiles on a 27-point stencil (4 dof) with its columns
    permuted at random: half-full 16x16 chunk tiles although the matrix's
    own 16x16 tiles are nearly empty; N not a multiple of 32 (slab edges),
    no long groups (no pieces).  Within the FP32 bound of the FP64 oracle."""
    A0 = bsp.gen_stencil27(8, 4, 13)
    perm = np.random.default_rng(3).permutation(A0.cols).astype(np.int32)
    rows = np.repeat(np.arange(A0.rows, dtype=np.int32), np.diff(A0.rowptr))
    nc = perm[A0.colidx]
    o = np.lexsort((nc, rows))
    A = bsp.HostCSR(A0.rows, A0.cols, A0.rowptr, np.ascontiguousarray(nc[o]), np.ascontiguousarray(A0.values[o]))
    vals_t, vals64, B_t, B64 = _case(A, N, "f16", 41)
    G = bsp.GatherTileMatrix(bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, vals64), dtype="f16")
    cpg = G.chunks_per_group()
    assert G.nsplit == 0 and A.nnz / (256.0 * cpg.sum()) > 0.4
    C = G.spmm(B_t.to(cuda)).cpu().numpy().astype(np.float64)
    G.check()
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    L = (16.0 * np.repeat(cpg, 16)[:A.rows] + 2.0)[:, None]
    u = 2.0 ** -24
    assert np.all(np.abs(C - Cref) <= 2.0 * (L * u / (1 - L * u)) * absC + 1e-30)
    G.free()


@pytest.mark.parametrize("engine,slab", [("slab", 0), ("slab", 16), ("grouped", 0)])
def test_spmm_split_rows_of_many_chunk_groups(cuda, engine, slab):
    """Split-row partials are summed in groups of up to 32 chunks and then per
    row: rows at the group boundaries (32, 33, 64, 65 chunks of 32 nonzeros)
    and one of 101 chunks, with alpha and beta, against the FP64 oracle;
    repeated calls give the same bits."""
    import torch
    rng = np.random.default_rng(77)
    rows, cols, N = 300, 4000, 32
    lens = rng.integers(0, 20, rows)
    for r, l in {3: 32 * 32, 50: 32 * 32 + 1, 120: 33 * 32, 200: 64 * 32, 201: 65 * 32 - 7, 299: 100 * 32 + 13}.items():
        lens[r] = l
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(cols, l, replace=False)) for l in lens]).astype(np.int32)
    A = bsp.HostCSR(rows, cols, rp, ci, rng.uniform(-1, 1, rp[-1]))
    vals_t, vals64, B_t, B64 = _case(A, N, "f16", 5)
    rpd, cid = _dev(cuda, A.rowptr, A.colidx)
    P = bsp.SpmmPlan(rpd, cid, vals_t.to(cuda), cols=cols, chunk=32)
    assert P._d.ngroups > P.nsplit   # some rows have several groups
    Bd = B_t.to(cuda)
    C1 = P.spmm(Bd, engine=engine, slab_cols=slab)
    assert torch.equal(C1, P.spmm(Bd, engine=engine, slab_cols=slab))
    Cref, absC = pyoracle.spmm_f64(A.rowptr, A.colidx, vals64, B64)
    assert np.all(np.abs(C1.cpu().numpy().astype(np.float64) - Cref) <= _tol(A, absC))
    Cin = rng.uniform(-1, 1, (rows, N)).astype(np.float32)
    Cd = torch.from_numpy(Cin.copy()).to(cuda)
    P.spmm(Bd, Cd, alpha=-2.0, beta=0.75, engine=engine, slab_cols=slab)
    want = -2.0 * Cref + 0.75 * Cin.astype(np.float64)
    assert np.all(np.abs(Cd.cpu().numpy().astype(np.float64) - want) <= _tol(A, absC, -2.0, Cin, 0.75))
    P.free()
