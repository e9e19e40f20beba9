"""GPU test of the allocation-free entry point.

gsmc_run_fb_blockwise_device_noalloc serves callers that cannot have the
library allocate device memory during a call: programs whose framework
allocator already holds the GPU's memory, services that cannot take the
device-wide synchronisation cudaMalloc/cudaFree may cause, and host
applications that load the library as a plug-in under their own
device-memory budget.  Its scratch is a fixed device array inside the library.

This file is named so that pytest collects it last: if it fails, a run that
stops at the first failure has already run every other test.  It builds all
its own state, so it passes alone in a fresh process as well as after the
rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, _lib, synthetic
from gamma_smc_cu_b200.infer import _estimate_scaled_params

pytestmark = pytest.mark.gpu

RTOL = 1e-4  # the posterior-mean tolerance the parity tests use
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")
FLAGS = _lib.GSMC_CI | _lib.GSMC_POSTERIOR


def _context():
    G, pos = synthetic.cohort("small")
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    return _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0), G.shape[1]


def _scratch_bytes(ctx):
    v = ctypes.c_uint64()
    _lib.check(_lib.load().gsmc_ctx_scratch_bytes(ctx.handle, ctypes.byref(v)))
    return v.value


def _run(fn, ctx, pi, pj, n_sites, core, flank, pad=3):
    import torch
    P = pi.numel()
    outs = [torch.full((n_sites, P + pad), -7.0, device=pi.device) for _ in KEYS]
    _lib.check(fn(ctx.handle, pi.data_ptr(), pj.data_ptr(), P, core, flank, FLAGS,
                  *[o.data_ptr() for o in outs], P + pad, pad, None))
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


def _assert_close(got, want):
    for k, g, w in zip(KEYS, got, want):
        rel = np.max(np.abs(g.astype(np.float64) - w) / np.maximum(np.abs(w), 1e-30))
        assert rel <= RTOL, (k, rel)
        assert np.array_equal(g, w), k


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    L = _lib.load()
    ctx, S = _context()
    dev = torch.device("cuda", ctx.device_id)
    pairs = synthetic.all_pairs(40)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    # two calls in a row with different windows: the second reuses the
    # scratch left by the first
    assert _scratch_bytes(ctx) == 0
    for core, flank in ((700, 300), (500, 100)):
        before = _scratch_bytes(ctx)
        got = _run(L.gsmc_run_fb_blockwise_device_noalloc, ctx, pi, pj, S, core, flank)
        assert _scratch_bytes(ctx) == before  # the call grew no context scratch
        want = _run(L.gsmc_run_fb_blockwise_device, ctx, pi, pj, S, core, flank)
        _assert_close(got, want)
        for g in got:
            assert (g[:, :3] == -7.0).all()  # columns outside out_col0.. untouched
    # and twice with identical arguments, back to back
    a = _run(L.gsmc_run_fb_blockwise_device_noalloc, ctx, pi, pj, S, S, 0)
    b = _run(L.gsmc_run_fb_blockwise_device_noalloc, ctx, pi, pj, S, S, 0)
    want = _run(L.gsmc_run_fb_blockwise_device, ctx, pi, pj, S, S, 0)
    _assert_close(a, want)
    _assert_close(b, want)
    # flanks (and cores) far beyond the sequence reach both ends, as they do in
    # the context path: both entry points clamp them to the sequence in int64
    for core, flank in ((700, 1 << 40), (1 << 40, 1 << 40)):
        got = _run(L.gsmc_run_fb_blockwise_device_noalloc, ctx, pi, pj, S, core, flank)
        want = _run(L.gsmc_run_fb_blockwise_device, ctx, pi, pj, S, core, flank)
        _assert_close(got, want)


def test_noalloc_rejects_core_beyond_scratch():
    import torch
    L = _lib.load()
    S = 140_000
    pos = np.arange(S, dtype=np.float64) * 7.0
    G = np.zeros((2, S), np.uint8)
    G[0, ::2] = 1
    G[1, 1::2] = 1
    ctx = _core.FlowContext(G, pos, 1e4, 1.25e-8, 1e-8, _core.DEFAULT_FLOW_FIELD, 0)
    dev = torch.device("cuda", ctx.device_id)
    pi = torch.tensor([1], dtype=torch.int32, device=dev)
    pj = torch.tensor([0], dtype=torch.int32, device=dev)
    out = torch.empty((S, 1), device=dev)
    with pytest.raises(ValueError, match="too large for the allocation-free"):
        _lib.check(L.gsmc_run_fb_blockwise_device_noalloc(
            ctx.handle, pi.data_ptr(), pj.data_ptr(), 1, S, 0, 0, out.data_ptr(), None, None,
            None, None, 1, 0, None))
