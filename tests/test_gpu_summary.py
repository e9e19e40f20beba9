"""Per-site summaries over pairs (run_fb_summary) on the GPU against the oracle
and the reference's own GPU build.

Tolerance: site_mean within 1e-6 relative of the oracle's float64 average of
its per-pair means (the kernel sums each warp's 32 means in float32 before the
float64 fold); site_min / site_max are selections of bit-exact per-pair means
and must match exactly.  The reference sums with float32 atomics in arbitrary
order, so its site_mean is checked at the 1e-4 bar; its site_min/site_max are
never written by its kernel (src/bindings.cpp:2725-2777) and are not compared.
"""
import os

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic

pytestmark = pytest.mark.gpu

NE = 1e4
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


@pytest.fixture(scope="module")
def small(small_data, oracle):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    return G, pos, mu, rho


def _check(got, want, rtol=1e-6):
    assert got["n_pairs"] == want["n_pairs"]
    assert _max_rel(got["site_mean"], want["site_mean"]) <= rtol
    assert np.array_equal(got["site_min"], want["site_min"])
    assert np.array_equal(got["site_max"], want["site_max"])


@pytest.mark.parametrize("width,ppt", [(128, 1), (32, 1), (128, 2), (32, 2)])
def test_summary_matches_oracle(small, oracle, flow_field, monkeypatch, width, ppt):
    G, pos, mu, rho = small
    monkeypatch.setenv("GSMC_SCAN_WIDTH", str(width))
    monkeypatch.setenv("GSMC_PAIRS_PER_THREAD", str(ppt))
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = [(i, j) for i in range(40) for j in range(i)][:-5]   # a partly filled warp
    want = oracle.run_fb_summary(G, pos, pairs, NE, mu, rho, flow_field)
    _check(ctx.run_fb_summary(pairs), want)
    # several pair passes, the last one partial, fold to the same result
    _check(ctx.run_fb_summary(pairs, pair_batch_size=96), want)
    # blockwise decode
    wantb = oracle.run_fb_summary(G, pos, pairs, NE, mu, rho, flow_field, core_block_sites=500,
                                  flank_sites=200)
    _check(ctx.run_fb_summary(pairs, core_block_sites=500, flank_sites=200), wantb)


def test_summary_edge_cases(small, oracle, flow_field):
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    assert ctx.run_fb_summary([])["site_mean"].shape == (0,)
    one = ctx.run_fb_summary([(7, 3)])
    m = ctx.run_fb([(7, 3)])["mean"][:, 0]
    assert np.array_equal(one["site_min"], m) and np.array_equal(one["site_max"], m)
    assert _max_rel(one["site_mean"], m) == 0.0
    with pytest.raises(ValueError, match="out of range"):
        ctx.run_fb_summary([(40, 0)])
    with pytest.raises(ValueError, match="pair_batch_size"):
        ctx.run_fb_summary([(1, 0)], pair_batch_size=0)


def test_summary_chromosome_slice_matches_full_output(oracle, flow_field):
    """356 haplotypes x 20k sites, 8,000 pairs: the summary equals the
    reduction of the full [S, P] mean output of the same decode."""
    G, pos = synthetic.cohort("chrom", n_sites=20000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = synthetic.random_pairs(356, 8000, 3)
    got = ctx.run_fb_summary(pairs, core_block_sites=8192, flank_sites=2048)
    full = ctx.run_fb_blockwise(pairs, core_block_sites=8192, flank_sites=2048,
                                pair_batch_size=-1)["mean"]
    assert _max_rel(got["site_mean"], full.astype(np.float64).mean(axis=1)) <= 1e-6
    assert np.array_equal(got["site_min"], full.min(axis=1))
    assert np.array_equal(got["site_max"], full.max(axis=1))


def test_summary_matches_reference_gpu_build(small, flow_field, ref_core):
    if ref_core is None:
        pytest.skip("reference _core not built in oracle/_ref")
    G, pos, mu, rho = small
    pairs = [(i, j) for i in range(40) for j in range(i)]
    want = ref_core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fb_summary(pairs)
    got = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fb_summary(pairs)
    assert want["n_pairs"] == got["n_pairs"]
    assert _max_rel(got["site_mean"], want["site_mean"]) <= 1e-4


def test_summary_of_few_pairs_over_long_windows(oracle, flow_field):
    """600 pairs over a 20,000-site window leave most of the GPU idle as
    summary tasks, so the per-pair means are decoded in exact speculative
    chunks and folded per site; same answer as the oracle, any pair batch."""
    import ctypes
    from gamma_smc_cu_b200 import _lib
    G, pos = synthetic.cohort("chrom", n_sites=20000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = [tuple(p) for p in synthetic.random_pairs(356, 600, 11)]
    got = ctx.run_fb_summary(pairs)
    launches = ctypes.c_int64()
    _lib.check(_lib.load().gsmc_ctx_spec_stats(ctx.handle, ctypes.byref(launches), None))
    assert launches.value >= 1            # the speculative per-pair path ran
    want = oracle.run_fb_summary(G, pos, pairs, NE, mu, rho, flow_field)
    _check(got, want)
    full = oracle.run_fb(G, pos, pairs, NE, mu, rho, flow_field, True, False)["mean"]
    assert np.array_equal(got["site_min"], full.min(axis=1))
    assert np.array_equal(got["site_max"], full.max(axis=1))
    batched = ctx.run_fb_summary(pairs, pair_batch_size=250)     # three pair batches
    assert _max_rel(batched["site_mean"], got["site_mean"]) <= 1e-6
    assert np.array_equal(batched["site_min"], got["site_min"])
    assert np.array_equal(batched["site_max"], got["site_max"])
