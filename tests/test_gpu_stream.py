"""Blockwise decoding streamed to a host sink (run_fb_blockwise_stream): the
units the sink receives reassemble exactly into run_fb_blockwise's arrays."""
import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic

pytestmark = pytest.mark.gpu

NE = 1e4
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def _collect(ctx, pairs, **kw):
    S, P = ctx.n_sites, len(pairs)
    got = {}
    seen = np.zeros((S, P), np.int32)

    def sink(s0, s1, p0, p1, outs):
        for k, v in outs.items():
            got.setdefault(k, np.full((S, P), np.nan, np.float32))[s0:s1, p0:p1] = v
        seen[s0:s1, p0:p1] += 1
        return False

    ctx.run_fb_blockwise_stream(pairs, sink, **kw)
    assert (seen == 1).all()  # every element delivered exactly once
    return got


def test_stream_equals_blockwise(small_data, oracle, flow_field):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = synthetic.all_pairs(40)
    want = ctx.run_fb_blockwise(pairs, core_block_sites=500, flank_sites=200,
                                pair_batch_size=-1, mean_only=False, return_posterior=True)
    # units of at most 300 pairs x 500 sites x 5 outputs: several pair chunks per window
    got = _collect(ctx, pairs, core_block_sites=500, flank_sites=200, mean_only=False,
                   return_posterior=True, max_chunk_bytes=500 * 300 * 5 * 4)
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k
    m = _collect(ctx, pairs[:77], core_block_sites=700, flank_sites=100, pair_batch_size=32)
    assert set(m) == {"mean"}
    wm = ctx.run_fb_blockwise(pairs[:77], core_block_sites=700, flank_sites=100,
                              pair_batch_size=-1)["mean"]
    assert np.array_equal(m["mean"], wm)


def test_stream_stop_and_errors(small_data, oracle, flow_field):
    G, pos = small_data
    ctx = _core.FlowContext(G, pos, NE, 1.25e-8, 1e-8, flow_field, 0)
    pairs = synthetic.all_pairs(40)
    calls = []

    def stop(s0, s1, p0, p1, outs):
        calls.append(s0)
        return True

    with pytest.raises(ValueError, match="stopped"):
        ctx.run_fb_blockwise_stream(pairs, stop, core_block_sites=500, flank_sites=100)
    assert len(calls) == 1

    def boom(*a):
        raise KeyError("sink failed")

    with pytest.raises(KeyError, match="sink failed"):
        ctx.run_fb_blockwise_stream(pairs, boom, core_block_sites=500, flank_sites=100)
    with pytest.raises(ValueError, match="out of range"):
        ctx.run_fb_blockwise_stream([(40, 1)], lambda *a: False)
    # the context still works after a stopped stream
    assert ctx.run_fb([(3, 1)])["mean"].shape == (G.shape[1], 1)


def test_stream_chromosome_slice(oracle, flow_field):
    G, pos = synthetic.cohort("chrom", n_sites=20000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = synthetic.random_pairs(356, 6000, 11)
    sums = np.zeros(20000)
    cols = {}

    def sink(s0, s1, p0, p1, outs):
        sums[s0:s1] += outs["mean"].astype(np.float64).sum(axis=1)
        for p in (0, 1234, 5999):
            if p0 <= p < p1:
                cols.setdefault(p, np.zeros(20000, np.float32))[s0:s1] = outs["mean"][:, p - p0]
        return False

    ctx.run_fb_blockwise_stream(pairs, sink, core_block_sites=8192, flank_sites=2048,
                                max_chunk_bytes=64 << 20)
    want = ctx.run_fb_blockwise(pairs, core_block_sites=8192, flank_sites=2048,
                                pair_batch_size=-1)["mean"]
    for p, col in cols.items():
        assert np.array_equal(col, want[:, p])
    assert np.allclose(sums, want.astype(np.float64).sum(axis=1), rtol=1e-9)
