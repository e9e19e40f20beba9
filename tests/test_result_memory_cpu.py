"""Host result arrays of the pageable mode, on the CPU.

Results of 64 MB or more are anonymous mappings advised MADV_HUGEPAGE (the
host copier's threads fault in every page of a fresh result as they fill
it); they must behave as plain float32 arrays: right shape, C order,
writable, 2 MB aligned, independent of each other, and freed with their last
view.  Smaller results stay np.empty arrays, and GSMC_HUGEPAGES=0 turns the
mapping off.
"""
import gc
import weakref

import numpy as np

from gamma_smc_cu_b200 import _core


def test_large_results_are_huge_page_mappings(monkeypatch):
    monkeypatch.setattr(_core, "_HUGEPAGES", True)
    monkeypatch.setattr(_core, "_RESULT_MEMORY", "pageable")
    shape = (1000, 17_000)                       # 68 MB
    a = _core._empty(shape)
    b = _core._empty(shape)
    assert a.shape == shape and a.dtype == np.float32
    assert a.flags["C_CONTIGUOUS"] and a.flags["WRITEABLE"]
    assert a.ctypes.data % (2 << 20) == 0
    a[:] = 1.0
    b[:] = 2.0
    assert float(a.sum()) == 1.0 * a.size and float(b[-1, -1]) == 2.0
    base = weakref.ref(a.base) if a.base is not None else None
    del a
    gc.collect()
    if base is not None:
        assert base() is None or base().closed


def test_small_results_and_switch(monkeypatch):
    monkeypatch.setattr(_core, "_RESULT_MEMORY", "pageable")
    monkeypatch.setattr(_core, "_HUGEPAGES", True)
    small = _core._empty((10, 10))
    assert small.base is None and small.shape == (10, 10)
    monkeypatch.setattr(_core, "_HUGEPAGES", False)
    big = _core._empty((1000, 17_000))
    assert big.base is None and big.dtype == np.float32
    empty = _core._empty((0, 5))
    assert empty.shape == (0, 5)


def test_mapping_failure_falls_back_to_np_empty(monkeypatch):
    import mmap

    def refuse(*a, **k):
        raise OSError(12, "Cannot allocate memory")

    monkeypatch.setattr(_core, "_HUGEPAGES", True)
    monkeypatch.setattr(_core, "_RESULT_MEMORY", "pageable")
    monkeypatch.setattr(mmap, "mmap", refuse)
    a = _core._empty((1000, 17_000))
    assert a.base is None and a.shape == (1000, 17_000) and a.dtype == np.float32
