"""libmvr loads and exports every entry point include/mvr.h declares; with no
GPU every entry point fails with an error status (never a CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mvr import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "mvr.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mvr_[a-z0-9_]+)\s*\(", txt)))


def test_header_lists_entry_points():
    syms = header_symbols()
    assert "mvr_search" in syms and "mvr_index_load" in syms
    assert set(syms) == set(_lib.EXPORTS)


def test_library_exports_every_symbol():
    L = _lib.lib()
    for s in header_symbols():
        assert hasattr(L, s), s


def test_elf_dynamic_symbols():
    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    for s in header_symbols():
        assert re.search(rf"\bT {s}$", out, re.M), s


def test_cli_binaries_built():
    for b in ("IGPGPUBasic", "IGPGPUPP"):
        assert os.access(os.path.join(_lib.LIB_DIR, b), os.X_OK)


@pytest.mark.skipif(_lib.lib().mvr_device_count() > 0, reason="GPU present")
def test_no_gpu_fails_loudly():
    L = _lib.lib()
    h = C.c_void_p()
    inv = np.array([2], np.uint32)
    cen = np.zeros((1, 128), np.float32)
    code = np.zeros(2, np.uint32)
    off = np.zeros(1, np.uint64)
    size = np.array([1], np.uint32)
    ids = np.zeros(1, np.uint32)
    w = np.zeros(4, np.float32)
    res = np.zeros(64, np.uint8)
    p = lambda a: C.c_void_p(a.ctypes.data)
    rc = L.mvr_index_from_arrays(p(inv), 1, p(cen), 1, 128, p(code), 2, p(off), p(size), p(ids), 1,
                                 p(w), 2, p(res), 0, C.byref(h))
    assert rc == _lib.MVR_ERR_CUDA
    assert b"no CUDA device" in L.mvr_last_error()
    rc = L.mvr_index_load(b"/nonexistent", 8, 2, 0, C.byref(h))
    assert rc == _lib.MVR_ERR_IO


def test_null_handle_errors():
    L = _lib.lib()
    st = _lib.Stats()
    rc = L.mvr_search(None, None, None, 1, 32, 10, 4, 100, 0, None, None, None, C.byref(st))
    assert rc == _lib.MVR_ERR_INVALID_ARG
    assert L.mvr_index_free(None) == 0
