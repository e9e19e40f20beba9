"""Speculative site-parallel chunks must not change a single bit.

When a call has too few (window, pair tile) tasks to fill the GPU, long
windows are decoded as parallel chunks with burn-in flanks; a verify kernel
compares the chunk boundary states bit for bit and re-decodes every pair
whose chunks did not join the exact trajectory.  These tests compare such
calls with the oracle's unchunked decode, exactly, with the default 2,048-site
flank and with a 4-site flank that forces many repairs.
"""
import ctypes

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, _lib, synthetic

pytestmark = pytest.mark.gpu

NE = 1e4
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def _stats(ctx):
    a, r = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.load().gsmc_ctx_spec_stats(ctx.handle, ctypes.byref(a), ctypes.byref(r)))
    return a.value, r.value


@pytest.fixture(scope="module")
def cohort(oracle, flow_field):
    G, pos = synthetic.cohort("chrom", n_sites=40000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    pairs = synthetic.random_pairs(356, 100, 21)
    want = oracle.run_fb(G, pos, [tuple(p) for p in pairs], NE, mu, rho, flow_field,
                         mean_only=False, return_posterior=True)
    return G, pos, mu, rho, pairs, want


def _check(got, want):
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("flank", [None, "4"])
def test_speculative_run_fb_is_exact(cohort, flow_field, monkeypatch, flank):
    G, pos, mu, rho, pairs, want = cohort
    if flank:
        monkeypatch.setenv("GSMC_SPEC_FLANK", flank)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    got = ctx.run_fb(pairs, mean_only=False, return_posterior=True)
    launches, repaired = _stats(ctx)
    assert launches >= 1
    if flank:
        assert repaired > 0  # a 4-site burn-in rarely joins: the repair path ran
    _check(got, want)
    # the per-query window path speculates the same way
    w = ctx.run_fb_window(pairs, 5000, 40000, mean_only=False, return_posterior=True)
    from oracle import oracle as O
    ww = O.fb_window(O.bitpack(G), pos, 5000, 35000, pairs[:, 0], pairs[:, 1], NE,
                     O.tables_for(flow_field, NE, mu, rho), ci=True, posterior=True)
    _check(w, ww)


def test_speculative_device_path_is_exact(cohort, flow_field, monkeypatch):
    import torch
    G, pos, mu, rho, pairs, want = cohort
    monkeypatch.setenv("GSMC_SPEC_FLANK", "16")
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    dev = torch.device("cuda", ctx.device_id)
    S, P = G.shape[1], len(pairs)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    outs = [torch.full((S, P), -1.0, device=dev) for _ in KEYS]
    _lib.check(_lib.load().gsmc_run_fb_blockwise_device(
        ctx.handle, pi.data_ptr(), pj.data_ptr(), P, S, 0, _lib.GSMC_CI | _lib.GSMC_POSTERIOR,
        *[o.data_ptr() for o in outs], P, 0, None))
    torch.cuda.synchronize()
    got = {k: o.cpu().numpy() for k, o in zip(KEYS, outs)}
    assert _stats(ctx)[1] > 0
    _check(got, want)


def test_speculation_off_and_full_gpu_untouched(cohort, flow_field, monkeypatch):
    G, pos, mu, rho, pairs, want = cohort
    monkeypatch.setenv("GSMC_SPECULATE", "0")
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    _check(ctx.run_fb(pairs, mean_only=False, return_posterior=True), want)
    assert _stats(ctx) == (0, 0)
    monkeypatch.delenv("GSMC_SPECULATE")
    # enough pairs to fill the GPU: no speculation
    many = synthetic.random_pairs(356, 20000, 5)
    ctx2 = _core.FlowContext(G[:, :9000], pos[:9000], NE, mu, rho, flow_field, 0)
    ctx2.run_fb_blockwise(many, core_block_sites=3000, flank_sites=1000, pair_batch_size=-1)
    assert _stats(ctx2)[0] == 0
