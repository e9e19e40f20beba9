"""Speculative chunks in a launch that fills the GPU twice over.

Such launches are cut only to keep chunks within the chunk cap (the
chromosome job's 32,768-site windows run as two chunks each).  Here the same
path runs on a small case: the chromosome-shape cohort's first 8,192 sites,
all 63,190 pairs, blockwise core 512 / flank 128 (16 windows x 247 two-pair
tiles = 3,952 tasks, over twice the resident tiles), with the chunk cap
lowered to 256 sites and the burn-in to 64 so every window is cut in two.
The whole output must equal, bit for bit, the same context's run with
speculation off, and sampled pairs must equal the oracle.
"""
import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, _lib, synthetic

pytestmark = pytest.mark.gpu

NE = 1e4
CORE, FLANK = 512, 128


def _run(ctx, G, pairs):
    import torch
    dev = torch.device("cuda", ctx.device_id)
    S, P = G.shape[1], len(pairs)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    out = torch.full((S, P), -1.0, device=dev)
    _lib.check(_lib.load().gsmc_run_fb_blockwise_device(
        ctx.handle, pi.data_ptr(), pj.data_ptr(), P, CORE, FLANK, 0, out.data_ptr(),
        None, None, None, None, P, 0, None))
    torch.cuda.synchronize()
    return out


def test_multiwave_launch_cut_to_the_chunk_cap(oracle, flow_field, monkeypatch):
    import torch
    G, pos = synthetic.cohort("chrom", n_sites=8192)
    pairs = synthetic.all_pairs(G.shape[0])
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)

    monkeypatch.setenv("GSMC_SPECULATE", "0")
    plain_ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    plain = _run(plain_ctx, G, pairs)
    assert plain_ctx.spec_stats()[0] == 0
    plain_ctx.close()

    monkeypatch.delenv("GSMC_SPECULATE")
    monkeypatch.setenv("GSMC_SPEC_MAX_CHUNK", "256")
    monkeypatch.setenv("GSMC_SPEC_FLANK", "64")
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    got = _run(ctx, G, pairs)
    launches, repairs = ctx.spec_stats()
    assert ctx.scan_shape() == (128, 2)
    assert launches == 1                      # the windows ran as speculative chunks
    assert torch.equal(got.view(torch.int32), plain.view(torch.int32))
    assert bool((got > 0).all())

    sel = np.sort(np.random.default_rng(7).choice(len(pairs), 32, replace=False))
    cols = got[:, torch.from_numpy(sel).to(got.device)].cpu().numpy()
    want = oracle.run_fb_blockwise(G, pos, [tuple(p) for p in pairs[sel]], NE, mu, rho,
                                   flow_field, CORE, FLANK, True, False)
    assert np.array_equal(cols.view(np.uint32),
                          np.ascontiguousarray(want["mean"], np.float32).view(np.uint32))
    ctx.close()
