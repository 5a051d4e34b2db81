"""The C ABI library loads and exports every symbol include/eacb200.h
declares (no GPU needed: nothing is called)."""
import ctypes
import os

import pytest

from masters_final_b200 import _lib


def test_header_symbols_exported():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libeacb200.so not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _lib.exported_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libeacb200.so not built")
    assert _lib.status_string(0) == "EACB_OK"
    assert _lib.status_string(-9) == "EACB_ERR_VALUE"


def test_workspace_sizes_are_monotone():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libeacb200.so not built")
    L = _lib.load()
    a = L.eacb_scan_workspace_size(1000)
    b = L.eacb_scan_workspace_size(10 ** 8)
    assert 0 < a < b
    assert L.eacb_boruvka_workspace_size(1000, 10000) < L.eacb_boruvka_workspace_size(10 ** 6, 10 ** 7)
