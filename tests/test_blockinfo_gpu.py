"""Device block statistics (bench/blockinfo.cpp:96-119) against the oracle
and the reference's own counts (fixture made by oracle/_ref/blockinfo)."""
import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


def test_blockinfo_matches_reference_fixture(cuda, golden):
    g = golden("blockinfo_ref.npz")
    mats = {"powerlaw": bsp.gen_powerlaw(30000, 2.0, 10000, 17), "laplace": bsp.gen_laplace2d(64, 80),
            "random": bsp.gen_random_bsr(1000, 4, 8, 0.3, 1.0, 5)}
    for i, name in enumerate(g["names"]):
        A = mats[str(name)]
        rp, ci = _dev(cuda, A.rowptr, A.colidx)
        r = bsp.blockinfo(rp, ci, rows=A.rows, cols=A.cols)
        assert r["blocks"] == int(g["blocks"][i]) and r["blocks_recorder"] == int(g["blocks_recorder"][i])


@pytest.mark.parametrize("n", [200000, 2000000])
def test_blockinfo_large_power_law(cuda, n):
    A = bsp.gen_powerlaw(n, 2.0, 10000, 23)
    rp, ci = _dev(cuda, A.rowptr, A.colidx)
    r = bsp.blockinfo(rp, ci, rows=A.rows, cols=A.cols)
    o = pyoracle.blockinfo(A.rowptr, A.colidx)
    assert r["blocks"] == o["blocks"] and r["blocks_recorder"] == o["blocks_recorder"]


def test_blockinfo_wrapped_key_collision(cuda):
    rows = 4 * 4295 + 1
    rp = np.zeros(rows + 1, np.int32)
    rp[1:] = 1
    rp[-1] = 2
    ci = np.array([4 * 54179, 0], np.int32)
    d = _dev(cuda, rp, ci)
    assert bsp.blockinfo(*d, rows=rows, cols=4 * 54179 + 4)["blocks"] == 1
