"""The C-ABI library loads and exports every symbol include/mfb.h declares
(no compute calls: runs on CPU-only hosts)."""
import ctypes
import os
import re

import pytest

from apogee_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mfb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mfb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert "mfb_create" in names and "mfb_hier_run" in names and "mfb_run_series" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmfb.so not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(L, name), name


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_error_mapping():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmfb.so not built")
    _lib.lib()
    with pytest.raises(ValueError):
        _lib.check(_lib.MFB_ERR_ARG)
    with pytest.raises(IndexError):
        _lib.check(_lib.MFB_ERR_INDEX)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.MFB_ERR_CUDA)
    assert _lib.check(3) == 3


def test_nbins_without_device():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libmfb.so not built")
    L = _lib.lib()
    assert L.mfb_nbins(4096, 256, 0, 4096) == 16
    assert L.mfb_nbins(4096, 17, 3, 4091) == (4088 + 16) // 17
    assert L.mfb_nbins(4096, 1000, 10, 99999) == 5
    assert L.mfb_nbins(4096, 0, 0, 10) == 0
    assert L.mfb_supported(4096) == 1 and L.mfb_supported(1000) == 0
