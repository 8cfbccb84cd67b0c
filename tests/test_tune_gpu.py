"""FP64 SpMV format autotuner: statistics, model choices, measured choices,
the structural-hash cache (in process and in a file), and the tuned executor
against the oracle."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import benchsp_b200 as bsp
from oracle import pyoracle

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _dev(cuda, *arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in arrs]


MATS = {
    "stencil": lambda: bsp.gen_stencil27(16, 4, 3),
    "powerlaw": lambda: bsp.gen_powerlaw(200000, 2.0, 10000, 4),
    "laplace": lambda: bsp.gen_laplace2d(300, 300),
    "randbsr8": lambda: bsp.gen_random_bsr(4096, 8, 6, 0.9, 1.0, 5),
}


@pytest.mark.parametrize("kind,fmt", [("stencil", "bsr"), ("powerlaw", "dasp"), ("laplace", "csr"),
                                      ("randbsr8", "bsr")])
def test_model_choice_and_executor(cuda, kind, fmt):
    bsp.tune_cache_clear()
    A = MATS[kind]()
    lens = np.diff(A.rowptr)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    r = bsp.tune_spmv(rp, ci, va, cols=A.cols)
    assert r["format_name"] == fmt and r["from_cache"] == 0
    assert r["max_len"] == lens.max() and r["long_rows"] == int(np.sum(lens >= 256))
    assert r["mean_len"] == pytest.approx(A.nnz / A.rows)
    if kind == "stencil":
        assert r["fill4"] == 1.0 and r["bs"] == 4
    if kind == "randbsr8":
        assert r["bs"] == 8 and r["fill8"] > 0.85
    x = bsp.gen_uniform(A.cols, 2)
    want = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    P = bsp.SpmvPlan(rp, ci, va, cols=A.cols)
    assert P.choice["format_name"] == fmt and P.choice["from_cache"] == 1
    (xd,) = _dev(cuda, x)
    y = P.spmv(xd).cpu().numpy()
    assert np.all(np.abs(y - want) <= tol)
    import torch
    y0 = torch.ones(A.rows, dtype=torch.float64, device=cuda)
    yb = P.spmv(xd, y0, alpha=2.0, beta=-1.0).cpu().numpy()
    assert np.all(np.abs(yb - (2.0 * want - 1.0)) <= 2 * tol + 4 * 2.0 ** -53 * (np.abs(2 * want) + 1))
    P.close()


def test_measured_choice_is_fastest_candidate_and_correct(cuda):
    bsp.tune_cache_clear()
    A = bsp.gen_powerlaw(100000, 1.8, 5000, 9)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    P = bsp.SpmvPlan(rp, ci, va, cols=A.cols, measure=True)
    c = P.choice
    assert c["spmv_us"] > 0 and c["from_cache"] == 0
    x = bsp.gen_uniform(A.cols, 3)
    (xd,) = _dev(cuda, x)
    want = pyoracle.spmv_f64(A.rowptr, A.colidx, A.values, x)
    tol = pyoracle.spmv_tolerance(A.rowptr, A.colidx, A.values, x)
    assert np.all(np.abs(P.spmv(xd).cpu().numpy() - want) <= tol)
    again = bsp.tune_spmv(rp, ci, va, cols=A.cols, measure=True)
    assert again["from_cache"] == 1 and again["format"] == c["format"] and again["lanes"] == c["lanes"]
    P.close()


def test_structural_key(cuda):
    A = bsp.gen_laplace2d(50, 60)
    rp, ci, va = _dev(cuda, A.rowptr, A.colidx, A.values)
    k = bsp.matrix_key(rp, ci, cols=A.cols)
    assert k == bsp.matrix_key(rp, ci, cols=A.cols)
    B = bsp.gen_laplace2d(60, 50)
    rpb, cib = _dev(cuda, B.rowptr, B.colidx)
    assert bsp.matrix_key(rpb, cib, cols=B.cols) != k
    # the values do not enter the key
    r1 = bsp.tune_spmv(rp, ci, va, cols=A.cols)
    r2 = bsp.tune_spmv(rp, ci, va * 3.0, cols=A.cols)
    assert r1["key"] == r2["key"] == k and r2["from_cache"] == 1


_CHILD = r"""
import sys, json
sys.path.insert(0, {root!r})
import torch, benchsp_b200 as bsp
A = bsp.gen_stencil27(12, 4, 1)
rp, ci, va = (torch.from_numpy(a).cuda() for a in (A.rowptr, A.colidx, A.values))
r = bsp.tune_spmv(rp, ci, va, cols=A.cols)
print(json.dumps({{"from_cache": r["from_cache"], "format": r["format"], "key": r["key"]}}))
"""


def test_cache_file_survives_processes(cuda, tmp_path):
    import json
    env = dict(os.environ, BSP_TUNE_CACHE=str(tmp_path / "tune.txt"))
    code = _CHILD.format(root=str(ROOT))
    a = json.loads(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                  check=True, timeout=300).stdout.strip().splitlines()[-1])
    b = json.loads(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                  check=True, timeout=300).stdout.strip().splitlines()[-1])
    assert a["from_cache"] == 0 and b["from_cache"] == 1
    assert a["format"] == b["format"] and a["key"] == b["key"]
    assert (tmp_path / "tune.txt").read_text().count("\n") == 1
