"""Uncached flow-field forward/backward (gamma_smc_flow_fb) on the GPU.

Against the reference's own GPU build it must be bit-identical (same float
arithmetic, same __exp10f/__log10f); against the CPU oracle, which uses libm
exp10f/log10f, within the 1e-4 relative tolerance.
"""
import numpy as np
import pytest

import gamma_smc_cu_b200 as G200
from gamma_smc_cu_b200 import _core, synthetic

pytestmark = pytest.mark.gpu

RTOL = 1e-4
KEYS = ("mean", "lower", "upper")


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


def test_flow_fb_matches_oracle(small_data, oracle, flow_field):
    G, pos = small_data
    pairs = [(i, j) for i in range(40) for j in range(i)]
    got = G200.gamma_smc_flow_fb(G, pos, pairs, Ne=1e4, flow_field_path=flow_field)
    want = oracle.flow_fb(G, pos, pairs, 1e4, 1.25e-8, 1e-8, flow_field)
    for k in KEYS:
        assert got[k].shape == want[k].shape == (G.shape[1], len(pairs))
        assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))
    m = G200.gamma_smc_flow_fb(G, pos, pairs[:30], Ne=1e4, flow_field_path=flow_field,
                               mean_only=True)
    assert set(m) == {"mean"} and np.array_equal(m["mean"], got["mean"][:, :30])


def test_flow_fb_other_rates_and_gaps(oracle, flow_field):
    rng = np.random.default_rng(8)
    gaps = rng.choice([0.0, 1.0, 7.0, 120.0, 999.0, 2500.0, 40000.0], size=500)
    pos = np.cumsum(gaps) + 3.0
    G = (rng.random((6, 500)) < 0.25).astype(np.uint8)
    pairs = [(i, j) for i in range(6) for j in range(i)]
    for Ne, mu, rho in ((1e4, 1.25e-8, 1e-8), (2e4, 2e-8, 5e-9), (5e3, 1e-8, 3e-8)):
        got = G200.gamma_smc_flow_fb(G, pos, pairs, Ne, mu, rho, flow_field)
        want = oracle.flow_fb(G, pos, pairs, Ne, mu, rho, flow_field)
        for k in KEYS:
            assert _max_rel(got[k], want[k]) <= RTOL, (Ne, k, _max_rel(got[k], want[k]))


def test_flow_fb_errors(small_data, flow_field, tmp_path):
    G, pos = small_data
    assert G200.gamma_smc_flow_fb(G, pos, [], flow_field_path=flow_field)["mean"].shape == \
        (G.shape[1], 0)
    with pytest.raises(ValueError, match="out of range"):
        G200.gamma_smc_flow_fb(G, pos, [(40, 0)], flow_field_path=flow_field)
    with pytest.raises(RuntimeError, match="flow field"):
        G200.gamma_smc_flow_fb(G, pos, [(1, 0)], flow_field_path=str(tmp_path / "missing.txt"))


def test_flow_fb_bit_exact_with_reference_gpu_build(small_data, flow_field, ref_core):
    if ref_core is None:
        pytest.skip("reference _core not built in oracle/_ref")
    G, pos = small_data
    pairs = [(i, j) for i in range(40) for j in range(i)]
    want = ref_core.gamma_smc_flow_fb(G, pos, pairs, 1e4, 1.25e-8, 1e-8, flow_field, False)
    got = G200.gamma_smc_flow_fb(G, pos, pairs, 1e4, 1.25e-8, 1e-8, flow_field, False)
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), (k, _max_rel(got[k], want[k]))


def _flow_fb_stats():
    import ctypes
    from gamma_smc_cu_b200 import _lib
    k, r = ctypes.c_int(), ctypes.c_int64()
    _lib.check(_lib.load().gsmc_flow_fb_stats(ctypes.byref(k), ctypes.byref(r)))
    return k.value, r.value


@pytest.mark.parametrize("flank", [None, "4"])
def test_flow_fb_speculative_site_chunks_are_exact(oracle, flow_field, ref_core, monkeypatch,
                                                   flank):
    """200 pairs over 20,000 sites are too few chains to fill the SMs, so the
    sites are cut into chunks whose forward and backward joins are checked
    bitwise; equal to the unchunked kernel bit for bit, also when a 4-site
    burn-in sends pairs to be decoded again whole."""
    G, pos = synthetic.cohort("chrom", n_sites=20000)
    pairs = [tuple(p) for p in synthetic.random_pairs(356, 200, 17)]
    monkeypatch.setenv("GSMC_SPECULATE", "0")
    plain = G200.gamma_smc_flow_fb(G, pos, pairs, Ne=1e4, flow_field_path=flow_field)
    assert _flow_fb_stats()[0] == 1
    monkeypatch.delenv("GSMC_SPECULATE")
    if flank:
        monkeypatch.setenv("GSMC_SPEC_FLANK", flank)
    got = G200.gamma_smc_flow_fb(G, pos, pairs, Ne=1e4, flow_field_path=flow_field)
    chunks, repaired = _flow_fb_stats()
    assert chunks > 1
    if flank:
        assert repaired > 0
    for k in KEYS:
        assert np.array_equal(got[k], plain[k]), k
    if not flank:
        want = oracle.flow_fb(G, pos, pairs, 1e4, 1.25e-8, 1e-8, flow_field)
        assert _max_rel(got["mean"], want["mean"]) <= RTOL
        if ref_core is not None:
            ref = ref_core.gamma_smc_flow_fb(G, pos, pairs, 1e4, 1.25e-8, 1e-8, flow_field, False)
            for k in KEYS:
                assert np.array_equal(got[k], ref[k]), k


def test_flow_fb_copy_wait_runs_out_then_recovers(small_data, flow_field):
    """A poll budget of 0 makes every CTA give up on its flow-field copy at
    once: the call reports GSMC_E_TIMEOUT (the CTAs still let their copies
    finish before exiting), and the next call on the same device, with the
    default budget back, is exact again."""
    import ctypes
    from gamma_smc_cu_b200 import _lib
    L = _lib.load()
    G, pos = small_data
    pairs = [(i, j) for i in range(12) for j in range(i)]
    want = G200.gamma_smc_flow_fb(G, pos, pairs, flow_field_path=flow_field, mean_only=True)
    prev = ctypes.c_int64()
    _lib.check(L.gsmc_set_copy_wait_polls(0, ctypes.byref(prev)))
    try:
        with pytest.raises(_lib.GsmcError, match="did not complete"):
            G200.gamma_smc_flow_fb(G, pos, pairs, flow_field_path=flow_field, mean_only=True)
    finally:
        _lib.check(L.gsmc_set_copy_wait_polls(prev.value, None))
    assert prev.value == 1 << 24
    got = G200.gamma_smc_flow_fb(G, pos, pairs, flow_field_path=flow_field, mean_only=True)
    assert np.array_equal(got["mean"], want["mean"])
    with pytest.raises(ValueError, match="non-negative"):
        _lib.check(L.gsmc_set_copy_wait_polls(-1, None))
