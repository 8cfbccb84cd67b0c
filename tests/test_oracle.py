"""The CPU oracle (oracle/liboracle.so) against the golden fixtures made by
the reference's own code (tests/golden/make_golden.py) and against scipy."""
import glob
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import pyoracle

GOLDEN = Path(__file__).resolve().parent / "golden"
SPMV = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "spmv_*.npz")))


@pytest.mark.parametrize("name", SPMV)
def test_spmv_fp64_bit_exact_with_reference(golden, name):
    g = golden(name)
    y = pyoracle.spmv_f64(g["rowptr"], g["colidx"], g["values"], g["x"])
    assert np.array_equal(y.view(np.uint64), g["y_fp64"].view(np.uint64))


@pytest.mark.parametrize("name", SPMV)
def test_spmv_fp32_bit_exact_with_reference(golden, name):
    g = golden(name)
    y = pyoracle.spmv_f32(g["rowptr"], g["colidx"], g["values"].astype(np.float32), g["x"].astype(np.float32))
    assert np.array_equal(y.view(np.uint32), g["y_fp32"].view(np.uint32))


@pytest.mark.parametrize("name", SPMV)
def test_spmv_fp16_bit_exact_with_reference(golden, name):
    g = golden(name)
    v16 = g["values"].astype(np.float32).astype(np.float16)
    x16 = g["x"].astype(np.float32).astype(np.float16)
    y = pyoracle.spmv_f16(g["rowptr"], g["colidx"], v16, x16).astype(np.float32)
    ref = g["y_fp16"]
    same = (y.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(y) & np.isnan(ref))
    assert same.all()


def test_half_conversion_matches_numpy():
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(50000) * 10.0 ** rng.integers(-8, 5, 50000)).astype(np.float32)
    L = pyoracle.orc()
    got = np.array([L.orc_f32_to_f16(float(a)) for a in v[:5000]], np.uint16)
    assert np.array_equal(got, v[:5000].astype(np.float16).view(np.uint16))


def _padded_scipy(rows, cols, rp, ci, va, bs):
    R = -(-rows // bs) * bs
    Cc = -(-cols // bs) * bs
    return sp.csr_matrix((va, ci, rp), shape=(rows, cols)).tocoo().tocsr(), R, Cc


@pytest.mark.parametrize("name", SPMV)
@pytest.mark.parametrize("bs", [4, 8])
def test_csr2bsr_oracle_against_scipy(golden, name, bs):
    g = golden(name)
    rows, cols = int(g["rows"]), int(g["cols"])
    o = pyoracle.csr2bsr(rows, cols, g["rowptr"], g["colidx"], g["values"], bs)
    R = -(-rows // bs) * bs
    Cc = -(-cols // bs) * bs
    M = sp.csr_matrix((g["values"], g["colidx"], g["rowptr"]), shape=(rows, cols))
    M = sp.vstack([sp.hstack([M, sp.csr_matrix((rows, Cc - cols))]), sp.csr_matrix((R - rows, Cc))]).tocsr()
    B = M.tobsr(blocksize=(bs, bs))
    B.sort_indices()
    assert np.array_equal(o["blcPtr"], B.indptr)
    assert np.array_equal(o["blcIdx"], B.indices)
    assert np.array_equal(o["blcVal"], B.data.reshape(-1))
    # bitmap = structural pattern of the CSR entries
    pat = sp.csr_matrix((np.ones_like(g["values"]), g["colidx"], g["rowptr"]), shape=(rows, cols))
    pat = sp.vstack([sp.hstack([pat, sp.csr_matrix((rows, Cc - cols))]), sp.csr_matrix((R - rows, Cc))]).tocsr()
    PB = pat.tobsr(blocksize=(bs, bs))
    PB.sort_indices()
    bits = (PB.data.reshape(-1, bs * bs) != 0) * (1 << np.arange(bs * bs, dtype=np.uint64))
    assert np.array_equal(o["blcMap"].astype(np.uint64), bits.sum(axis=1).astype(np.uint64))
    assert o["rowPtrbyWarp"][-1] == o["warpnum"]


AMGT = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "amgt_*.npz")))


@pytest.mark.parametrize("name", AMGT)
def test_csr2bsr_oracle_against_reference_gpu_capture(golden, name):
    g = golden(name)
    rows, cols = int(g["rows"]), int(g["cols"])
    o = pyoracle.csr2bsr(rows, cols, g["rowptr"], g["colidx"], g["values"], 4)
    for k in ("blcPtr", "blcIdx", "blcVal", "blcMap", "rowPtrbyWarp", "rowIdxbyWarp"):
        assert np.array_equal(o[k], g[k]), k
    assert o["warpnum"] == int(g["warpnum"]) and o["blc_num"] == int(g["blc_num"])
    assert abs(o["stand"] - float(g["stand"])) <= 1e-6 * max(1.0, float(g["stand"]))


DBSR = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "dbsr_*.npz")))


@pytest.mark.parametrize("name", DBSR)
def test_dbsr_oracle_against_reference(golden, name):
    g = golden(name)
    rec = name.endswith("_rec.npz")
    o = pyoracle.csr2dbsr(g["rowptr"], g["colidx"], g["values"], rec)
    if rec:
        for k in ("rec_rowptr", "rec_colidx", "rec_values"):
            assert np.array_equal(o[k], g[k]), k
    assert o["blc_row"] == int(g["blc_row"]) and o["blocknnz"] == int(g["blocknnz"])
    assert np.array_equal(o["blcPtr"], g["blcPtr"])
    assert np.array_equal(o["colIdx"], g["colIdx_d"])
    assert np.array_equal(o["blcVal"], g["blcVal"])
    assert np.array_equal(o["blcMap"], g["blcMap"])
    in_bounds = bool(int(g["balance_in_bounds"]))
    assert o["balance_overflow"] == (0 if in_bounds else 1)
    if in_bounds:
        assert o["warpnum"] == int(g["warpnum"])
        assert np.array_equal(o["prefix"], g["prefix"])
        if rec:
            assert np.array_equal(o["recorderMap"], g["recorderMap"])


BCSR = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "bcsr_*.npz")))


@pytest.mark.parametrize("name", BCSR)
def test_bcsr_oracle_against_reference(golden, name):
    g = golden(name)
    o = pyoracle.csr2bcsr(int(g["rows"]), int(g["cols"]), g["rowptr"], g["colidx"], g["values"],
                          int(g["tile_m"]), int(g["tile_k"]))
    assert o["nonzeroBlocks"] == int(g["nonzeroBlocks"])
    assert o["rowRegions"] == int(g["rowRegions"]) and o["colRegions"] == int(g["colRegions"])
    for k in ("bcsrRowPtr", "bcsrColIdx", "bcsrVal", "mapping"):
        assert np.array_equal(o[k], g[k]), k


DASP = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "dasp_*.npz")))
DASP_ARRS = ("long_val", "long_cid", "long_ptr_warp", "reg_val", "reg_cid", "block_ptr", "irreg_val", "irreg_cid",
             "irreg_rpt", "short_val", "short_cid", "order_rid")
DASP_INTS = ("row_long", "row_block", "blocknum", "short_row_1", "common_13", "short_row_34", "short_row_2",
             "offset_reg", "offset_short1", "offset_short13", "offset_short34", "offset_short22",
             "fill0_nnz_short13", "fill0_nnz_short34")


@pytest.mark.parametrize("name", DASP)
def test_dasp_oracle_against_reference_capture(golden, name):
    g = golden(name)
    o = pyoracle.dasp_pack(g["rowptr"], g["colidx"], g["values"], float(g["threshold"]), int(g["block_longest"]))
    for k in DASP_ARRS:
        ref = g.get("arr_" + k, np.zeros(0))
        assert np.array_equal(o[k], ref), k
    for k in DASP_INTS:
        assert o[k] == int(g["int_" + k]), k
    assert o["block_num_all"] == int(g["int_grid_all"])


@pytest.mark.parametrize("n,alpha,cap,th,bl", [(60000, 2.0, 10000, 0.75, 256), (20000, 1.6, 3000, 0.5, 64)])
def test_dasp_oracle_against_live_reference(n, alpha, cap, th, bl):
    """Runs the reference's spmv_all packing (oracle/_ref/dasp_capture) on a
    larger seeded power-law matrix when it has been built."""
    if not (pyoracle.REF_DIR / "dasp_capture").exists():
        pytest.skip("oracle/_ref/dasp_capture not built")
    rng = np.random.default_rng(n)
    lens = np.minimum(rng.zipf(alpha, n), cap)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, int(L), replace=False)) for L in lens]).astype(np.int32)
    va = rng.standard_normal(ci.size)
    rec = pyoracle.run_capture("dasp_capture", n, n, rp, ci, va, np.zeros(n), th, bl)
    o = pyoracle.dasp_pack(rp, ci, va, th, bl)
    ints = {"long_ptr_warp", "reg_cid", "block_ptr", "irreg_cid", "irreg_rpt", "short_cid", "long_cid", "order_rid"}
    for k in DASP_ARRS:
        dt = np.int32 if k in ints else np.float64
        assert np.array_equal(o[k], np.frombuffer(rec.get("arr:" + k, b""), dt)), k


def _bi_matrices():
    import benchsp_b200 as bsp
    yield "powerlaw", bsp.gen_powerlaw(30000, 2.0, 10000, 17)
    yield "laplace", bsp.gen_laplace2d(64, 80)
    yield "random", bsp.gen_random_bsr(1000, 4, 8, 0.3, 1.0, 5)


@pytest.mark.parametrize("name", ["powerlaw", "laplace", "random"])
def test_blockinfo_oracle_against_live_reference(name):
    """bench/blockinfo.cpp compiled from the reference (oracle/_ref/blockinfo)."""
    if not (pyoracle.REF_DIR / "blockinfo").exists():
        pytest.skip("oracle/_ref/blockinfo not built")
    A = dict(_bi_matrices())[name]
    ref = pyoracle.run_ref_blockinfo(A.rows, A.cols, A.rowptr, A.colidx, A.values)
    assert pyoracle.blockinfo(A.rowptr, A.colidx) == ref


def test_blockinfo_oracle_against_fixture(golden):
    import benchsp_b200 as bsp
    g = golden("blockinfo_ref.npz")
    for i, name in enumerate(g["names"]):
        A = dict(_bi_matrices())[str(name)]
        o = pyoracle.blockinfo(A.rowptr, A.colidx)
        assert o["blocks"] == int(g["blocks"][i]) and o["blocks_recorder"] == int(g["blocks_recorder"][i])


def test_blockinfo_wrapped_keys_collide_like_the_reference():
    """row/4*1000005 wraps in 32 bits: rows 4*4295 apart with block columns
    54179 apart share a key, so the reference counts one block for two."""
    rows = 4 * 4295 + 1
    rp = np.zeros(rows + 1, np.int32)
    rp[1:] = 1  # row 0 has one entry, rows 1.. none except the last
    rp[-1] = 2
    ci = np.array([4 * 54179, 0], np.int32)
    o = pyoracle.blockinfo(rp, ci)
    assert o["blocks"] == 1


def test_cpu_cg_oracle_converges():
    import benchsp_b200 as bsp
    A = bsp.gen_poisson3d(10)
    b = bsp.gen_uniform(A.rows, 3)
    x, it = pyoracle.cg(A.rowptr, A.colidx, A.values, b, 1e-10)
    assert 0 < it < 500
    assert pyoracle.rel_residual(A.rowptr, A.colidx, A.values, b, x) <= 1e-10


def test_scaled_bsr_oracle_known_answers_and_round_trip():
    """orc_bsr_scale: a block whose largest magnitude is 1.0 gets e = -14
    (FP16, 1.0 -> q = 2^14 = 0x7400) or e = 0 (BF16, q = 0x3F80); an all-zero
    block e = 0; the dequantized values are within half an ulp of the 16-bit
    type (relative 2^-11 / 2^-8 of the block's largest magnitude)."""
    from oracle import pyoracle
    blk = np.zeros(16)
    blk[0] = 1.0
    blk[5] = -0.5
    vals = np.concatenate([blk, np.zeros(16)])
    idx = np.array([3, 7], np.int32)
    key, val, bad = pyoracle.bsr_scale(idx, vals, 4, "f16")
    assert bad == 0 and list(key) == [3 | ((128 - 14) << 24), 7 | (128 << 24)]
    assert val[0] == 0x7400 and val[5] == 0xF000 and not val[16:].any()
    key, val, _ = pyoracle.bsr_scale(idx, vals, 4, "bf16")
    assert list(key >> 24) == [128, 128] and val[0] == 0x3F80 and val[5] == 0xBF00
    rng = np.random.default_rng(3)
    for bs, dt, rel in ((4, "f16", 2.0 ** -11), (8, "f16", 2.0 ** -11), (4, "bf16", 2.0 ** -8), (8, "bf16", 2.0 ** -8)):
        nb = 500
        v = rng.standard_normal(nb * bs * bs) * np.repeat(10.0 ** rng.integers(-30, 30, nb), bs * bs)
        key, val, bad = pyoracle.bsr_scale(np.arange(nb, dtype=np.int32), v, bs, dt)
        assert bad == 0
        back = pyoracle.bsr_unscale(key, val, bs, dt).reshape(nb, -1)
        m = np.abs(v.reshape(nb, -1)).max(axis=1, keepdims=True)
        assert np.all(np.abs(back - v.reshape(nb, -1)) <= rel * np.maximum(np.abs(v.reshape(nb, -1)), 2.0 ** -14 * m))
    # tile layout of an 8x8 block: tile (r//4, c//4), entry (r%4, c%4)
    v = np.arange(64, dtype=np.float64) + 1
    key, val, _ = pyoracle.bsr_scale(np.zeros(1, np.int32), v, 8, "bf16")
    back = pyoracle.bsr_unscale(key, val, 8, "bf16")
    assert np.array_equal(back, v)    # small integers are exact in BF16 after a power-of-two scale
    e = int(key[0] >> 24) - 128
    q = np.array([np.ldexp(float(i + 1), -e) for i in range(64)], np.float32).view(np.uint32) >> 16
    assert val[16 * 1 + 0] == q[4] and val[16 * 2 + 0] == q[32] and val[16 * 3 + 5] == q[36 + 9]


def test_oracle_bsr_spmv_helper_matches_csr_spmv():
    from oracle import pyoracle
    import benchsp_b200 as bsp
    A = bsp.gen_random_bsr(40, 4, 5, 0.3, 1.0, 2)
    o = pyoracle.csr2bsr(A.rows, A.cols, A.rowptr, A.colidx, A.values, 4)
    x = bsp.gen_uniform(A.cols, 5)
    y, ay = pyoracle.bsr_spmv_f64(A.rows, o["blcPtr"], o["blcIdx"], o["blcVal"], 4, x)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    assert np.allclose(y, ref, rtol=1e-13, atol=1e-13)
    assert np.allclose(ay, pyoracle.abs_rowsum(A.rowptr, A.colidx, A.values, x), rtol=1e-13)
