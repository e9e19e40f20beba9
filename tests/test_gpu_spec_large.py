"""Parity at the benchmarked shapes, on sampled pairs.

* One 50,000-site window (the full-posterior slice of the chromosome-shape
  cohort) over 8,192 pairs, mean + alpha + beta in HBM through the
  device-resident entry point: the call is cut into exact speculative site
  chunks (2,048-site burn-ins), once in the shape the planner picks and once
  forced to two pairs per thread.  256 sampled pairs are compared with the
  oracle bit for bit; every pair is checked through the identity
  mean = alpha / max(beta, 1e-10) * 2 Ne that the combine computes in float32.
* The 2,000-haplotype cohort (genotype rows 2,000 wide) on a 20,000-site
  prefix, 4,096 random pairs, blockwise core 8,192 / flank 2,048 as the
  large-cohort stream runs it; 64 sampled pairs against the oracle.
"""
import ctypes

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, _lib, synthetic

pytestmark = pytest.mark.gpu

NE = 1e4
KEYS = ("mean", "posterior_alpha", "posterior_beta")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def slice50k(oracle):
    G, pos = synthetic.cohort("chrom", n_sites=50_000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    pairs = synthetic.random_pairs(356, 8192, 31)
    return G, pos, mu, rho, pairs


@pytest.mark.parametrize("ppt", [None, "2"])
def test_50k_window_8192_pairs_speculative(slice50k, oracle, flow_field, monkeypatch, ppt):
    import torch
    G, pos, mu, rho, pairs = slice50k
    if ppt:
        monkeypatch.setenv("GSMC_PAIRS_PER_THREAD", ppt)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    dev = torch.device("cuda", ctx.device_id)
    S, P = G.shape[1], len(pairs)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    outs = {k: torch.full((S, P), -1.0, device=dev) for k in KEYS}
    _lib.check(_lib.load().gsmc_run_fb_blockwise_device(
        ctx.handle, pi.data_ptr(), pj.data_ptr(), P, S, 2048, _lib.GSMC_POSTERIOR,
        outs["mean"].data_ptr(), None, None, outs["posterior_alpha"].data_ptr(),
        outs["posterior_beta"].data_ptr(), P, 0, None))
    torch.cuda.synchronize()
    launches, _ = ctx.spec_stats()
    assert launches == 1                      # the window ran as speculative chunks
    if ppt:
        assert ctx.scan_shape() == (128, 2)
    sel = np.sort(np.random.default_rng(32).choice(P, 256, replace=False))
    st = torch.from_numpy(sel).to(dev)
    got = {k: o[:, st].cpu().numpy() for k, o in outs.items()}
    want = oracle.run_fb_blockwise(G, pos, [tuple(p) for p in pairs[sel]], NE, mu, rho,
                                   flow_field, S, 2048, True, True)
    for k in KEYS:
        assert np.array_equal(_bits(got[k]), _bits(want[k])), k
    # every pair: the stored mean is the combine of the stored alpha and beta
    rows = torch.arange(0, S, 53, device=dev)
    m, a, b = (outs[k][rows].cpu().numpy() for k in KEYS)
    recon = (a / np.maximum(b, np.float32(1e-10))) * np.float32(2.0 * NE)
    assert recon.dtype == np.float32
    assert np.array_equal(_bits(recon), _bits(m))
    assert (m > 0).all() and np.isfinite(m).all()


def test_2000_haplotype_cohort_blockwise(oracle, flow_field):
    import torch
    G, pos = synthetic.cohort("cohort", n_sites=20_000)
    assert G.shape[0] == 2000
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    pairs = synthetic.random_pairs(2000, 4096, 33)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    dev = torch.device("cuda", ctx.device_id)
    S, P = G.shape[1], len(pairs)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    out = torch.full((S, P), -1.0, device=dev)
    _lib.check(_lib.load().gsmc_run_fb_blockwise_device(
        ctx.handle, pi.data_ptr(), pj.data_ptr(), P, 8192, 2048, 0, out.data_ptr(), None, None,
        None, None, P, 0, None))
    torch.cuda.synchronize()
    sel = np.sort(np.random.default_rng(34).choice(P, 64, replace=False))
    got = out[:, torch.from_numpy(sel).to(dev)].cpu().numpy()
    want = oracle.run_fb_blockwise(G, pos, [tuple(p) for p in pairs[sel]], NE, mu, rho,
                                   flow_field, 8192, 2048, True, False)
    assert np.array_equal(_bits(got), _bits(want["mean"]))
    # the highest haplotype indices are exercised
    assert int(pairs.max()) >= 1990
