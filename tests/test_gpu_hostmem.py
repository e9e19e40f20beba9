"""Host result memory: page-locked result buffers written by the DMA directly.

set_result_memory("pinned") makes the host result arrays of FlowContext calls
views of page-locked buffers from the library's cache; the copier sees a
page-locked destination and lets the device-to-host DMA write it directly.
The values must be the same bits as with ordinary (pageable) arrays, and
buffers must come back to the cache for the next call.
"""
import ctypes
import gc

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, _lib

pytestmark = pytest.mark.gpu

KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def test_pinned_results_equal_pageable(small_data, flow_field):
    G, pos = small_data
    pairs = [(i, j) for i in range(40) for j in range(i)]
    ctx = _core.FlowContext(G, pos, 1e4, 1.25e-8, 1e-8, flow_field, 0)
    want = ctx.run_fb_blockwise(pairs, core_block_sites=700, flank_sites=300, mean_only=False,
                                return_posterior=True)
    prev = _core.set_result_memory("pinned")
    try:
        for _ in range(3):   # buffers are released and reused call after call
            got = ctx.run_fb_blockwise(pairs, core_block_sites=700, flank_sites=300,
                                       mean_only=False, return_posterior=True)
            for k in KEYS:
                assert got[k].dtype == np.float32 and got[k].shape == want[k].shape
                assert np.array_equal(got[k], want[k]), k
            del got
            gc.collect()
        r = ctx.run_fb(pairs[:100], mean_only=True)
        _core.set_result_memory("pageable")
        assert np.array_equal(r["mean"], ctx.run_fb(pairs[:100])["mean"])
    finally:
        _core.set_result_memory(prev)
    with pytest.raises(ValueError):
        _core.set_result_memory("managed")
    ctx.close()


def test_host_alloc_cache_roundtrip():
    L = _lib.load()
    p = ctypes.c_void_p()
    _lib.check(L.gsmc_host_alloc(1 << 20, ctypes.byref(p)))
    first = p.value
    _lib.check(L.gsmc_host_free(ctypes.c_void_p(first)))
    _lib.check(L.gsmc_host_alloc((1 << 20) - 100, ctypes.byref(p)))
    assert p.value == first                    # the cached block fits: reused
    _lib.check(L.gsmc_host_free(p))
    with pytest.raises(ValueError, match="not a gsmc_host_alloc buffer"):
        _lib.check(L.gsmc_host_free(ctypes.c_void_p(first + 64)))
    _lib.check(L.gsmc_host_cache_limit(0))     # frees the cache
    _lib.check(L.gsmc_host_cache_limit(256 << 30))
