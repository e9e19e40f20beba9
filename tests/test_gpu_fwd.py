"""Forward-only (filtered) posterior, run_fwd, on the GPU.

The reference runs it on a float16 copy of its hom multi-step table with the
device's __exp10f/__log10f (src/kernels/gamma_smc_flow.cu:1136-1256).  The
CUDA path uses the same arithmetic, so against the reference's own GPU build
it must be bit-identical; the CPU oracle uses libm exp10f/log10f, which differ
by a few ulp, so it is held to the 1e-4 relative tolerance.
"""
import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic

pytestmark = pytest.mark.gpu

RTOL = 1e-4
NE = 1e4


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


@pytest.fixture(scope="module")
def small(small_data, oracle):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    return G, pos, mu, rho


def test_fwd_matches_oracle(small, oracle, flow_field):
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = [(i, j) for i in range(40) for j in range(i)]
    got = ctx.run_fwd(pairs, mean_only=False)
    want = oracle.run_fwd(G, pos, pairs, NE, mu, rho, flow_field, mean_only=False)
    for k in ("mean", "lower", "upper"):
        assert got[k].shape == (G.shape[1], len(pairs)) and got[k].dtype == np.float32
        assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))
    m = ctx.run_fwd(pairs[:50])
    assert set(m) == {"mean"} and np.array_equal(m["mean"], got["mean"][:, :50])
    assert ctx.run_fwd([])["mean"].shape == (G.shape[1], 0)
    with pytest.raises(ValueError, match="out of range"):
        ctx.run_fwd([(40, 1)])


def test_fwd_gap_edges(oracle, flow_field):
    """Zero gaps (repeated positions), gaps of exactly 1000 and 2000 bp, gaps
    beyond the 1000-step table, half-integer positions."""
    rng = np.random.default_rng(4)
    gaps = np.array([0.0, 0.4, 0.5, 1.5, 999.0, 1000.0, 1001.0, 2000.0, 2500.5, 15000.0, 3.0] * 30)
    pos = np.cumsum(rng.permutation(gaps)) + 10.0
    G = (rng.random((8, len(pos))) < 0.3).astype(np.uint8)
    G[0, ::3] = 1
    pairs = [(i, j) for i in range(8) for j in range(i)]
    ctx = _core.FlowContext(G, pos, NE, 1.25e-8, 1e-8, flow_field, 0)
    got = ctx.run_fwd(pairs, mean_only=False)
    want = oracle.run_fwd(G, pos, pairs, NE, 1.25e-8, 1e-8, flow_field, mean_only=False)
    for k in ("mean", "lower", "upper"):
        assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))


def test_fwd_bit_exact_with_reference_gpu_build(small, flow_field, ref_core):
    if ref_core is None:
        pytest.skip("reference _core not built in oracle/_ref")
    G, pos, mu, rho = small
    pairs = [(i, j) for i in range(40) for j in range(i)]
    want = ref_core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fwd(pairs, False)
    got = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fwd(pairs, mean_only=False)
    for k in ("mean", "lower", "upper"):
        assert np.array_equal(got[k], want[k]), (k, _max_rel(got[k], want[k]))


def test_fwd_chromosome_slice(oracle, flow_field):
    G, pos = synthetic.cohort("chrom", n_sites=10000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = synthetic.random_pairs(356, 3000, 5)
    got = ctx.run_fwd(pairs)["mean"]
    sel = np.random.default_rng(0).choice(3000, 40, replace=False)
    want = oracle.run_fwd(G, pos, [tuple(p) for p in pairs[sel]], NE, mu, rho, flow_field)["mean"]
    assert _max_rel(got[:, sel], want) <= RTOL


def _spec_stats(ctx):
    import ctypes
    from gamma_smc_cu_b200 import _lib
    la, rep = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.load().gsmc_ctx_spec_stats(ctx.handle, ctypes.byref(la), ctypes.byref(rep)))
    return la.value, rep.value


@pytest.mark.parametrize("flank", [None, "4"])
def test_fwd_speculative_site_chunks_are_exact(oracle, flow_field, ref_core, monkeypatch, flank):
    """300 pairs over 40,000 sites fill few SMs as one chain per pair, so the
    sites are cut into chunks with burn-ins whose joins are checked bitwise;
    the result equals the unchunked kernel's bit for bit, also when a 4-site
    burn-in makes most pairs fail the check and be decoded again whole."""
    G, pos = synthetic.cohort("chrom", n_sites=40000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    pairs = [tuple(p) for p in synthetic.random_pairs(356, 300, 13)]
    monkeypatch.setenv("GSMC_SPECULATE", "0")
    plain = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fwd(pairs, mean_only=False)
    monkeypatch.delenv("GSMC_SPECULATE")
    if flank:
        monkeypatch.setenv("GSMC_SPEC_FLANK", flank)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    got = ctx.run_fwd(pairs, mean_only=False)
    launches, repaired = _spec_stats(ctx)
    assert launches >= 1
    if flank:
        assert repaired > 0
    for k in ("mean", "lower", "upper"):
        assert np.array_equal(got[k], plain[k]), k
    want = oracle.run_fwd(G, pos, pairs, NE, mu, rho, flow_field, mean_only=True)
    assert _max_rel(got["mean"], want["mean"]) <= RTOL
    if ref_core is not None and not flank:
        ref = ref_core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fwd(pairs, True)
        assert np.array_equal(got["mean"], ref["mean"])
