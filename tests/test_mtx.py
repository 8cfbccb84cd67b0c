"""Matrix Market reader/writer: triplets and values against scipy.io.mmread
(scipy's reader is fast_matrix_market, the library the reference's drivers
read through), values against Python's correctly rounded float(), CSR
against a stable lexsort of the triplets (the reference's conversion,
bench/spmvfp64.cpp:56-86, with a stable order among duplicates), thread-count
invariance, write/read round trips, and the error cases.  The GPU test
checks the device-built CSR against the host one, bit for bit."""
import warnings

import numpy as np
import pytest
import scipy.io

import benchsp_b200 as bsp

pytestmark = pytest.mark.filterwarnings("ignore::DeprecationWarning")


def _mmread(path):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return scipy.io.mmread(str(path))


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return p


def _stable_csr(rows, r, c, v):
    o = np.lexsort((c, r))          # stable: equal (row, col) keep triplet order
    rp = np.zeros(rows + 1, np.int64)
    np.add.at(rp, r.astype(np.int64) + 1, 1)
    return np.cumsum(rp).astype(np.int32), c[o], v[o]


CASES = {
    "general": """%%MatrixMarket matrix coordinate real general
% a comment
4 5 6
1 1 1.5
4 5 -2.25e-3
2 3 7
3 1 1e300
4 5 0.1
1 2 -0.0
""",
    "symmetric_crlf_comments": "%%MatrixMarket matrix coordinate real symmetric\r\n%c\r\n\r\n3 3 4\r\n"
                               "1 1 2.0\r\n2 1 -1.0\r\n3 2 -1.5 extra\r\n\r\n  3 3 4.0\r\n\r\n",
    "out_of_range": """%%MatrixMarket matrix coordinate real general
2 2 4
1 1 1e400
2 2 1e-400
1 2 -1e400
2 1 -4e-330
""",
    "skew": """%%MatrixMarket matrix coordinate real skew-symmetric
3 3 2
2 1 1.25
3 1 -4
""",
    "hermitian_real": """%%MatrixMarket matrix coordinate real hermitian
2 2 2
1 1 3
2 1 0.5
""",
    "pattern_symmetric": """%%MatrixMarket matrix coordinate pattern symmetric
4 4 4
1 1
2 1
4 2
4 4
""",
    "integer": """%%MatrixMarket matrix coordinate integer general
2 3 3
1 3 -17
2 1 9007199254740993
2 2 0
""",
    "digits_and_ranges": """%%MatrixMarket matrix coordinate real general
3 3 9
1 1 3.14159265358979323846264338327950288
1 2 2.2250738585072011e-308
1 3 4.9406564584124654e-324
2 1 1.7976931348623157e308
2 2 0.30000000000000000000000000000000000000000001
2 3 9007199254740993
3 1 -1.000000000000000000000000000000000001E-5
3 2 123456789012345678901234567890e-20
3 3 .5e1
""",
    "array_general": """%%MatrixMarket matrix array real general
2 3
1
2
0
4
5.5
-6
""",
    "array_symmetric": """%%MatrixMarket matrix array real symmetric
3 3
1
2
3
4
5
6
""",
    "array_skew": """%%MatrixMarket matrix array real skew-symmetric
3 3
1
2
3
""",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_triplets_match_scipy_mmread(tmp_path, name):
    p = _write(tmp_path, name + ".mtx", CASES[name])
    f = bsp.MtxFile(p)
    r, c, v = f.triplets()
    ref = _mmread(p)
    if f.format == "array":
        dense = np.zeros((f.rows, f.cols))
        dense[r, c] = v
        assert np.array_equal(_bits(dense), _bits(np.asarray(ref, np.float64)))
        return
    assert np.array_equal(r, ref.row) and np.array_equal(c, ref.col), (r, ref.row, c, ref.col)
    assert np.array_equal(_bits(v), _bits(ref.data.astype(np.float64)))
    assert (f.rows, f.cols) == ref.shape


def test_values_are_correctly_rounded(tmp_path):
    rng = np.random.default_rng(11)
    toks = []
    for _ in range(20000):
        nd = int(rng.integers(1, 30))
        digits = "".join(str(d) for d in rng.integers(0, 10, nd))
        point = int(rng.integers(0, nd + 1))
        m = digits[:point] + "." + digits[point:]
        e = int(rng.integers(-340, 320))
        sign = "-" if rng.random() < 0.5 else ""
        toks.append(f"{sign}{m}e{e}")
    # halfway cases between neighbouring doubles, written out exactly
    for _ in range(2000):
        x = float(rng.uniform(0.5, 2.0)) * 10.0 ** int(rng.integers(-300, 300))
        nxt = np.nextafter(x, np.inf)
        from decimal import Decimal, getcontext
        getcontext().prec = 800
        mid = (Decimal(x) + Decimal(float(nxt))) / 2
        toks.append(format(mid, "f") if 1e-30 < abs(x) < 1e30 else format(mid, "e"))
    n = len(toks)
    body = "".join(f"{k + 1} 1 {t}\n" for k, t in enumerate(toks))
    p = _write(tmp_path, "vals.mtx", f"%%MatrixMarket matrix coordinate real general\n{n} 1 {n}\n{body}")
    r, c, v = bsp.MtxFile(p).triplets()
    want = np.array([float(t) for t in toks])
    assert np.array_equal(_bits(v), _bits(want))
    assert np.array_equal(_bits(v), _bits(_mmread(p).data))


def test_csr_matches_stable_sort_of_triplets(tmp_path):
    rng = np.random.default_rng(5)
    n, m = 3000, 40000
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    r[:500] = r[500:1000]        # duplicates (row, col) with different values
    c[:500] = c[500:1000]
    v = rng.standard_normal(m)
    body = "".join(f"{a + 1} {b + 1} {float(x)!r}\n" for a, b, x in zip(r, c, v))
    p = _write(tmp_path, "dup.mtx", f"%%MatrixMarket matrix coordinate real general\n{n} {n} {m}\n{body}")
    A = bsp.read_mtx(p)
    rp, ci, va = _stable_csr(n, r.astype(np.int32), c.astype(np.int32), v)
    assert np.array_equal(A.rowptr, rp) and np.array_equal(A.colidx, ci)
    assert np.array_equal(_bits(A.values), _bits(va))


def test_comment_lines_inside_the_body_are_skipped(tmp_path):
    # fast_matrix_market rejects these; this reader skips them like blank lines
    p = _write(tmp_path, "c.mtx", "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n% note\n"
                                  "   % indented note\n2 2 3\n")
    r, c, v = bsp.MtxFile(p).triplets()
    assert np.array_equal(r, [0, 1]) and np.array_equal(v, [1.0, 3.0])


def test_symmetric_expansion_and_fmm_diag_zero(tmp_path):
    p = _write(tmp_path, "s.mtx", CASES["symmetric_crlf_comments"])
    f = bsp.MtxFile(p)
    assert (f.entries, f.nnz, f.symmetry) == (4, 6, "symmetric")
    g = bsp.MtxFile(p, fmm_diag_zero=True)
    assert g.nnz == 2 * g.entries
    r, c, v = g.triplets()
    assert np.array_equal(r[4:], [0, 0, 1, 2]) and np.array_equal(c[4:], [0, 1, 2, 2])
    assert np.array_equal(v[4:], [0.0, -1.0, -1.5, 0.0])
    A = g.csr_host()
    # the explicit zero follows its diagonal entry; the matrix is unchanged
    assert np.array_equal(A.rowptr, [0, 3, 5, 8])
    assert np.array_equal(A.values[:3], [2.0, 0.0, -1.0])


def test_expansion_flags_and_buffer_entry(tmp_path):
    import ctypes as C
    text = CASES["skew"].encode()
    p = _write(tmp_path, "k.mtx", CASES["skew"])
    assert bsp.MtxFile(p, flags=bsp._lib.MTX_NO_EXPAND).nnz == 2
    s = bsp.MtxFile(_write(tmp_path, "s.mtx", CASES["symmetric_crlf_comments"]), flags=bsp._lib.MTX_DIAG_DUPLICATE)
    r, c, v = s.triplets()
    assert np.array_equal(v[4:], [2.0, -1.0, -1.5, 4.0]) and s.nnz == 8
    with pytest.raises(bsp.BspError):
        bsp.MtxFile(p, flags=bsp._lib.MTX_DIAG_DUPLICATE | bsp._lib.MTX_DIAG_ZERO)
    with pytest.raises(bsp.BspError):
        bsp.MtxFile(p, flags=64)
    h = C.c_void_p()
    bsp._lib.check(bsp.lib().bsp_mtx_read_buffer(text, len(text), 0, 2, C.byref(h)))
    info = bsp._lib.BspMtxInfo()
    bsp._lib.check(bsp.lib().bsp_mtx_get_info(h, C.byref(info)))
    assert (info.rows, info.entries, info.nnz, info.symmetry) == (3, 2, 4, 2)
    v2 = np.empty(4)
    bsp._lib.check(bsp.lib().bsp_mtx_triplets(h, None, None, v2.ctypes.data_as(C.c_void_p)))
    assert np.array_equal(v2, [1.25, -4.0, -1.25, 4.0])
    bsp.lib().bsp_mtx_free(h)


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_thread_count_does_not_change_the_result(tmp_path, threads):
    A = bsp.gen_powerlaw(60000, 1.7, 3000, 2)
    p = tmp_path / "big.mtx"
    bsp.write_mtx(p, A, threads=5)
    f = bsp.MtxFile(p, threads=threads)
    r, c, v = f.triplets()
    rows = np.repeat(np.arange(A.rows, dtype=np.int32), np.diff(A.rowptr))
    assert np.array_equal(r, rows) and np.array_equal(c, A.colidx)
    assert np.array_equal(_bits(v), _bits(A.values))
    B = f.csr_host()
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.colidx, A.colidx)


def test_column_major_file_gives_row_major_csr(tmp_path):
    A = bsp.gen_powerlaw(20000, 1.8, 500, 6)
    r = np.repeat(np.arange(A.rows), np.diff(A.rowptr))
    o = np.lexsort((r, A.colidx))
    body = "".join(f"{a + 1} {b + 1} {float(x)!r}\n" for a, b, x in zip(r[o], A.colidx[o], A.values[o]))
    p = _write(tmp_path, "cm.mtx", f"%%MatrixMarket matrix coordinate real general\n{A.rows} {A.cols} {A.nnz}\n{body}")
    B = bsp.read_mtx(p, threads=4)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.colidx, A.colidx)
    assert np.array_equal(_bits(B.values), _bits(A.values))


def test_write_read_round_trip_is_exact(tmp_path):
    rng = np.random.default_rng(3)
    A = bsp.gen_stencil27(6, 3, 4)
    vals = rng.standard_normal(A.nnz) * 10.0 ** rng.integers(-300, 300, A.nnz)
    vals[::97] = 5e-324
    vals[::89] = -0.0
    A = bsp.HostCSR(A.rows, A.cols, A.rowptr, A.colidx, vals)
    p = tmp_path / "rt.mtx"
    bsp.write_mtx(p, A)
    B = bsp.read_mtx(p)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.colidx, A.colidx)
    assert np.array_equal(_bits(B.values), _bits(A.values))
    ref = _mmread(p).tocsr()
    assert np.array_equal(_bits(np.sort(ref.data)), _bits(np.sort(A.values)))
    q = tmp_path / "pat.mtx"
    bsp.write_mtx(q, A, pattern=True)
    P = bsp.read_mtx(q)
    assert np.array_equal(P.colidx, A.colidx) and np.all(P.values == 1.0)


def test_empty_matrix(tmp_path):
    p = _write(tmp_path, "e.mtx", "%%MatrixMarket matrix coordinate real general\n3 2 0\n")
    A = bsp.read_mtx(p)
    assert A.rows == 3 and A.nnz == 0 and np.array_equal(A.rowptr, [0, 0, 0, 0])


BAD = {
    "no_banner": ("3 3 1\n1 1 1\n", bsp._lib.BSP_ERR_INVALID),
    "complex": ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 2\n", bsp._lib.BSP_ERR_UNSUPPORTED),
    "vector": ("%%MatrixMarket vector coordinate real general\n1 1 1\n1 1 1\n", bsp._lib.BSP_ERR_UNSUPPORTED),
    "too_few": ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 1\n", bsp._lib.BSP_ERR_INVALID),
    "too_many": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n2 2 1\n", bsp._lib.BSP_ERR_INVALID),
    "row_range": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", bsp._lib.BSP_ERR_INVALID),
    "col_zero": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 0 1\n", bsp._lib.BSP_ERR_INVALID),
    "plus_sign": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 +1\n", bsp._lib.BSP_ERR_INVALID),
    "banner_case": ("%%MATRIXMARKET matrix coordinate real general\n1 1 1\n1 1 1\n", bsp._lib.BSP_ERR_INVALID),
    "bad_value": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 x\n", bsp._lib.BSP_ERR_INVALID),
    "no_size": ("%%MatrixMarket matrix coordinate real general\n% only comments\n", bsp._lib.BSP_ERR_INVALID),
    "nonsquare_sym": ("%%MatrixMarket matrix coordinate real symmetric\n2 3 1\n1 1 1\n", bsp._lib.BSP_ERR_INVALID),
    "array_pattern": ("%%MatrixMarket matrix array pattern general\n1 1\n", bsp._lib.BSP_ERR_INVALID),
}


@pytest.mark.parametrize("name", sorted(BAD))
def test_malformed_files_are_rejected(tmp_path, name):
    text, status = BAD[name]
    p = _write(tmp_path, name + ".mtx", text)
    with pytest.raises(bsp.BspError) as e:
        bsp.MtxFile(p)
    assert e.value.status == status


def test_missing_file_is_rejected(tmp_path):
    with pytest.raises(bsp.BspError):
        bsp.MtxFile(tmp_path / "nope.mtx")


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["powerlaw_dups", "symmetric", "row_sorted", "col_major"])
def test_device_csr_matches_host_csr(cuda, tmp_path, kind):
    import torch
    if kind in ("row_sorted", "col_major"):
        A = bsp.gen_powerlaw(100000, 1.8, 4000, 4)
        p = tmp_path / "o.mtx"
        r = np.repeat(np.arange(A.rows), np.diff(A.rowptr))
        o = np.arange(A.nnz) if kind == "row_sorted" else np.lexsort((r, A.colidx))
        body = "".join(f"{a + 1} {b + 1} {float(x)!r}\n" for a, b, x in zip(r[o], A.colidx[o], A.values[o]))
        p.write_text(f"%%MatrixMarket matrix coordinate real general\n{A.rows} {A.cols} {A.nnz}\n{body}")
    elif kind == "symmetric":
        A = bsp.gen_poisson3d(40)
        keep = np.repeat(np.arange(A.rows), np.diff(A.rowptr)) >= A.colidx     # lower triangle
        r = np.repeat(np.arange(A.rows), np.diff(A.rowptr))[keep]
        body = "".join(f"{a + 1} {b + 1} {float(x)!r}\n" for a, b, x in zip(r, A.colidx[keep], A.values[keep]))
        p = _write(tmp_path, "sym.mtx",
                   f"%%MatrixMarket matrix coordinate real symmetric\n{A.rows} {A.rows} {keep.sum()}\n{body}")
    else:
        A = bsp.gen_powerlaw(200000, 1.8, 5000, 9)
        p = tmp_path / "pl.mtx"
        bsp.write_mtx(p, A)
        # append duplicates of the first rows' entries so equal keys occur
        lines = p.read_text().splitlines()
        extra = lines[2:2002]
        head = lines[1].split()
        lines[1] = f"{head[0]} {head[1]} {int(head[2]) + len(extra)}"
        p.write_text("\n".join(lines + [e.rsplit(" ", 1)[0] + " 0.5" for e in extra]) + "\n")
    f = bsp.MtxFile(p)
    H = f.csr_host()
    rp, ci, va = f.csr(cuda)
    torch.cuda.synchronize()
    assert np.array_equal(rp.cpu().numpy(), H.rowptr) and np.array_equal(ci.cpu().numpy(), H.colidx)
    assert np.array_equal(_bits(va.cpu().numpy()), _bits(H.values))
    if kind != "powerlaw_dups":
        assert np.array_equal(H.rowptr, A.rowptr) and np.array_equal(H.colidx, A.colidx)
        assert np.array_equal(_bits(H.values), _bits(A.values))


PROBE = r"""
#include <cstdio>
#include <fstream>
#include "fast_matrix_market/fast_matrix_market.hpp"
int main(int argc, char **argv) {
  struct { int64_t nrows = 0, ncols = 0; std::vector<int32_t> rows, cols; std::vector<double> vals; } t;
  std::ifstream f(argv[1]);
  fast_matrix_market::read_options o;
  if (argc > 2) o.generalize_symmetry = false;
  fast_matrix_market::read_matrix_market_triplet(f, t.nrows, t.ncols, t.rows, t.cols, t.vals, o);
  printf("%lld %lld %zu\n", (long long)t.nrows, (long long)t.ncols, t.vals.size());
  for (size_t k = 0; k < t.vals.size(); ++k) printf("%d %d %a\n", t.rows[k], t.cols[k], t.vals[k]);
}
"""


def test_fast_matrix_market_dropin_header(tmp_path):
    """The reference drivers' read_matrix_market_triplet call, compiled
    against the library's drop-in header, returns the library's triplets
    (with fast_matrix_market's explicit zero per mirrored diagonal)."""
    import shutil
    import subprocess
    from pathlib import Path
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "probe.cpp"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    libdir = root / "benchsp_b200" / "lib"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{root / 'benchsp_b200' / 'compat'}", f"-I{root / 'include'}",
                    str(src), "-o", str(exe), f"-L{libdir}", "-lbspmv", f"-Wl,-rpath,{libdir}"], check=True)
    p = _write(tmp_path, "s.mtx", CASES["symmetric_crlf_comments"])
    for flag, fmm in ((["x"], None), ([], True)):
        out = subprocess.run([str(exe), str(p), *flag], capture_output=True, text=True, check=True).stdout.split("\n")
        rows, cols, n = map(int, out[0].split())
        trip = [ln.split() for ln in out[1:1 + n]]
        r = np.array([int(a) for a, _, _ in trip])
        c = np.array([int(b) for _, b, _ in trip])
        v = np.array([float.fromhex(x) for _, _, x in trip])
        if fmm:
            rr, cc, vv = bsp.MtxFile(p, fmm_diag_zero=True).triplets()
        else:
            rr, cc, vv = (a[:4] for a in bsp.MtxFile(p).triplets())   # stored entries only
        assert (rows, cols) == (3, 3)
        assert np.array_equal(r, rr) and np.array_equal(c, cc) and np.array_equal(_bits(v), _bits(vv))
