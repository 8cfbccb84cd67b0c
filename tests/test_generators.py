"""Seeded synthetic inputs: sizes of the benchmark configurations (at small
scale), determinism and CSR well-formedness."""
import numpy as np

import benchsp_b200 as bsp


def well_formed(A):
    rp, ci = A.rowptr, A.colidx
    assert rp[0] == 0 and rp[-1] == ci.size
    assert np.all(np.diff(rp) >= 0)
    for r in range(0, A.rows, max(1, A.rows // 97)):
        seg = ci[rp[r]:rp[r + 1]]
        assert np.all(np.diff(seg) > 0)
        assert seg.size == 0 or (seg[0] >= 0 and seg[-1] < A.cols)


def test_laplace2d_matches_closed_form():
    A = bsp.gen_laplace2d(512, 512)
    assert A.rows == 262144 and A.nnz == 1308672
    well_formed(A)
    assert np.all(np.diff(A.rowptr) <= 5)
    d = A.values[A.colidx == np.repeat(np.arange(A.rows), np.diff(A.rowptr))]
    assert np.all(d == 4.0)


def test_poisson3d_size():
    A = bsp.gen_poisson3d(16)
    assert A.rows == 4096 and A.nnz == 7 * 4096 - 6 * 256
    well_formed(A)


def test_stencil27_block_count():
    A = bsp.gen_stencil27(10, 4, 3)
    assert A.rows == 4000 and A.nnz == 16 * 28 ** 3
    well_formed(A)


def test_generators_are_deterministic():
    a = bsp.gen_powerlaw(20000, 2.0, 10000, 9)
    b = bsp.gen_powerlaw(20000, 2.0, 10000, 9)
    assert np.array_equal(a.colidx, b.colidx) and np.array_equal(a.values, b.values)
    well_formed(a)
    assert 4.0 < a.nnz / a.rows < 8.0
    c = bsp.gen_powerlaw(20000, 2.0, 10000, 10)
    assert not np.array_equal(a.rowptr, c.rowptr)


def test_random_bsr_fill():
    A = bsp.gen_random_bsr(500, 4, 16, 0.3, 1.0, 4)
    well_formed(A)
    fill = A.nnz / (500 * 16 * 16)
    assert 0.55 < fill < 0.75


def test_uniform_range():
    x = bsp.gen_uniform(100000, 1)
    assert x.min() >= -1 and x.max() <= 1 and abs(x.mean()) < 0.02


def test_oracle_generator_is_bit_identical_to_the_library():
    """bench.py's reference arm builds the headline matrix with the oracle's
    copy of the generator (so it never loads the library): same arrays, bit
    for bit, as the library's generator, on a grid with boundary and interior
    nodes and at the headline's seeds."""
    import hashlib

    from oracle import pyoracle
    seed = 20261203 + 1
    for m, dof in ((7, 4), (12, 2), (5, 1)):
        A = bsp.gen_stencil27(m, dof, seed)
        rp, ci, va = pyoracle.gen_stencil27(m, dof, seed)
        h = [hashlib.sha256(a.tobytes()).hexdigest() for a in (A.rowptr, A.colidx, A.values)]
        assert h == [hashlib.sha256(a.tobytes()).hexdigest() for a in (rp, ci, va)]
    x = bsp.gen_uniform(123457, seed + 1)
    assert np.array_equal(x.view(np.uint64), pyoracle.gen_uniform(123457, seed + 1).view(np.uint64))
