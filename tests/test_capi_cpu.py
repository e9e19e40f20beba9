"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import numpy as np
import pytest

from gamma_smc_cu_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(REPO, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(gsmc_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = _declared()
    for must in ("gsmc_ctx_create", "gsmc_ctx_destroy", "gsmc_run_fb", "gsmc_run_fb_blockwise",
                 "gsmc_mem_info", "gsmc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert _declared() <= set(_lib.SIGNATURES)


def test_version_and_error_string():
    L = _lib.load()
    assert b"sm_100a" in L.gsmc_version()
    assert isinstance(_lib.last_error(), str)


def test_host_side_validation_without_gpu():
    """Argument errors are caught on the host and reported as ValueError."""
    L = _lib.load()
    n = ctypes.c_int64()
    with pytest.raises(ValueError, match="core_block_sites"):
        _lib.check(L.gsmc_block_count(100, 0, ctypes.byref(n)))
    _lib.check(L.gsmc_block_count(100, 30, ctypes.byref(n)))
    assert n.value == 4
    _lib.check(L.gsmc_block_count(0, 30, ctypes.byref(n)))
    assert n.value == 0
    with pytest.raises(ValueError, match="null context"):
        _lib.check(L.gsmc_ctx_info(None, None, None, None))
    with pytest.raises(ValueError, match="65535"):
        _lib.check(L.gsmc_bitpack(None, 70000, 10, None))
