"""The C-ABI library loads, exports every entry point include/*.h declares,
and rejects bad arguments with a status (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

import benchsp_b200 as bsp
from benchsp_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_in_headers():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(bsp_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = bsp.lib()
    names = declared_in_headers()
    assert names, "no declarations found"
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    # every declared symbol has a ctypes prototype
    assert declared_in_headers() <= set(_lib.declared_symbols())


def test_version_string():
    assert b"sm_100a" in bsp.lib().bsp_version()


def test_invalid_arguments_are_reported():
    L = bsp.lib()
    st = L.bsp_csr_spmv(-1, 0, 0, None, None, None, 0, None, None, 1.0, 0.0, 0, 0, None)
    assert st == _lib.BSP_ERR_INVALID
    assert b"negative" in L.bsp_last_error()
    st = L.bsp_csr_spmv(4, 4, 4, None, None, None, 0, None, None, 1.0, 0.0, 0, 0, None)
    assert st == _lib.BSP_ERR_INVALID
    st = L.bsp_csr_spmv(4, 4, 4, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), 0, C.c_void_p(16),
                        C.c_void_p(16), 1.0, 0.0, 0, 3, None)
    assert st == _lib.BSP_ERR_INVALID and b"lanes_per_row" in L.bsp_last_error()
    d = _lib.BspBsr()
    assert L.bsp_csr2bsr(4, 4, 0, C.c_void_p(16), None, None, 5, C.byref(d), None) == _lib.BSP_ERR_INVALID
    with pytest.raises(bsp.BspError):
        _lib.check(_lib.BSP_ERR_INVALID)


def test_zero_rows_is_a_no_op():
    L = bsp.lib()
    assert L.bsp_csr_spmv(0, 0, 0, None, None, None, 0, None, None, 1.0, 0.0, 0, 0, None) == _lib.BSP_OK


def test_merge_workspace_size_monotone():
    a = bsp.csr_merge_workspace_bytes(1000, 5000)
    b = bsp.csr_merge_workspace_bytes(100000, 500000)
    assert 0 < a < b
