"""Device CSR->BCSR (bit-exact with csrToBcsr, utils/utils.hpp:10) and the
generic tile SpMV against the oracle."""
import glob
from pathlib import Path

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
BCSR = sorted(Path(p).name for p in glob.glob(str(GOLDEN / "bcsr_*.npz")))


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


@pytest.mark.parametrize("name", BCSR)
def test_csr2bcsr_bit_exact_with_reference_fixture(cuda, golden, name):
    g = golden(name)
    rows, cols, tm, tk = int(g["rows"]), int(g["cols"]), int(g["tile_m"]), int(g["tile_k"])
    rp, ci, va = _dev(cuda, g["rowptr"], g["colidx"], g["values"])
    B = bsp.csr2bcsr(rp, ci, va, rows=rows, cols=cols, tile_m=tm, tile_k=tk, mapping=True)
    a = B.arrays()
    assert B.nonzeroBlocks == int(g["nonzeroBlocks"])
    assert B.rowRegions == int(g["rowRegions"]) and B.colRegions == int(g["colRegions"])
    for k in ("bcsrRowPtr", "bcsrColIdx", "bcsrVal", "mapping"):
        assert np.array_equal(a[k], g[k]), k


@pytest.mark.parametrize("tm,tk", [(2, 2), (3, 3), (4, 4), (16, 16), (16, 8), (8, 16), (1, 7)])
def test_csr2bcsr_generated_and_spmv(cuda, tm, tk):
    A = bsp.gen_powerlaw(20000, 2.0, 3000, 21)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    B = bsp.csr2bcsr(rp, ci, va, rows=A.rows, cols=A.cols, tile_m=tm, tile_k=tk)
    o = pyoracle.csr2bcsr(A.rows, A.cols, A.rowptr, A.colidx, A.values, tm, tk, with_mapping=False)
    a = B.arrays()
    for k in ("bcsrRowPtr", "bcsrColIdx", "bcsrVal"):
        assert np.array_equal(a[k], o[k]), k
    x = bsp.gen_uniform(A.cols, 4)
    ref = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    y = B.spmv(_dev(cuda, x)[0]).cpu().numpy()
    assert np.all(np.abs(y - ref) <= pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x))
