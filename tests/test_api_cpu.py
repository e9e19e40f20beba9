"""API contract of infer / infer_blockwise without a GPU.

Restates the argument-validation, fake-context and mocked-memory tests of the
reference (tests/unit/test_infer.py:323-352, 354-422, 444-593, 666-675): the
wrapper must forward exactly these arguments, emit these warnings and raise
these errors, looking ``_core.FlowContext`` / ``_core.cuda_mem_info`` up at
call time.
"""
import numpy as np
import pytest

import gamma_smc_cu_b200
from gamma_smc_cu_b200 import synthetic


@pytest.fixture(autouse=True)
def host_het_counts(monkeypatch):
    """infer() makes its calibration counts on the GPU; without one, the
    oracle's host counts stand in (the GPU tests check they are identical)."""
    from oracle import oracle as O
    monkeypatch.setattr(gamma_smc_cu_b200._core, "diploid_het_counts",
                        lambda G: O.diploid_het_counts(G))


@pytest.fixture(scope="module")
def genotype_data():
    pos = synthetic.positions_for(177, 1.0e5, 42)
    G = synthetic.haplotypes(20, pos, 43)
    return G, pos


def _fake_ctx(pos, calls=None, captured=None):
    class FakeFlowContext:
        def __init__(self, G, positions, Ne, mu, rho, flow_field_path, cache_steps):
            if calls is not None:
                calls["init"] = dict(shape=G.shape, positions=len(positions), Ne=Ne, mu=mu,
                                     rho=rho, flow_field_path=flow_field_path,
                                     cache_steps=cache_steps)

        def run_fb_blockwise(self, pairs, core_block_sites, flank_sites, pair_batch_size,
                             max_streams, mean_only, return_posterior=False):
            kw = dict(pairs=list(pairs), core_block_sites=core_block_sites,
                      flank_sites=flank_sites, pair_batch_size=pair_batch_size,
                      max_streams=max_streams, mean_only=mean_only,
                      return_posterior=return_posterior)
            if calls is not None:
                calls["run"] = kw
            if captured is not None:
                captured.update(kw)
            return {"mean": np.ones((len(pos), len(pairs)), np.float32),
                    "blocks": np.array([[0, len(pos), 0, len(pos)]], np.int32)}

        def run_fb(self, pairs, mean_only=True, return_posterior=False):
            if calls is not None:
                calls["run_fb"] = dict(pairs=list(pairs), mean_only=mean_only,
                                       return_posterior=return_posterior)
            return {"mean": np.ones((len(pos), len(pairs)), np.float32)}
    return FakeFlowContext


def test_requires_explicit_pairs(genotype_data):
    G, pos = genotype_data
    with pytest.raises(ValueError, match="explicit pairs"):
        gamma_smc_cu_b200.infer_blockwise(G, pos, flow_field_path="dummy-flow-field.txt")


@pytest.mark.parametrize("kw,match,exc", [
    (dict(pair_batch_size=0), "pair_batch_size", ValueError),
    (dict(pair_batch_size=-2), "pair_batch_size", ValueError),
    (dict(max_streams=0), "max_streams", ValueError),
    (dict(flank_sites=-1), "flank_sites", ValueError),
    (dict(core_block_sites="not-a-number"), "core_block_sites", TypeError),
    (dict(core_block_sites=0), "core_block_sites", ValueError),
    (dict(core_block_sites=10, flank_sites=0), "flank_sites=0", ValueError),
    (dict(return_posterior=True, max_streams=2, core_block_sites=10**6, flank_sites=0),
     "return_posterior", ValueError),
])
def test_blockwise_argument_validation(genotype_data, kw, match, exc):
    G, pos = genotype_data
    with pytest.raises(exc, match=match):
        gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=[(0, 1)],
                                          flow_field_path="dummy-flow-field.txt", **kw)


def test_rejects_mismatched_positions(genotype_data):
    G, pos = genotype_data
    with pytest.raises(ValueError, match="positions length"):
        gamma_smc_cu_b200.infer(G, pos[:-1], pairs=[(0, 1)])
    with pytest.raises(ValueError, match="positions is required"):
        gamma_smc_cu_b200.infer(G)
    with pytest.raises(ValueError, match="2D"):
        gamma_smc_cu_b200.infer(G[0], pos)


def test_passes_blockwise_args(monkeypatch, genotype_data):
    G, pos = genotype_data
    pairs = [(0, 1), (2, 3)]
    calls = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, calls=calls))
    r = gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=pairs, flow_field_path="dummy-flow-field.txt",
                                          core_block_sites=256, flank_sites=64,
                                          pair_batch_size=32, max_streams=3, mean_only=False)
    assert r["mean"].shape == (len(pos), len(pairs))
    assert r["pairs"] == pairs
    np.testing.assert_array_equal(r["positions"], pos)
    np.testing.assert_array_equal(r["blocks"], np.array([[0, len(pos), 0, len(pos)]], np.int32))
    assert calls["init"]["shape"] == G.shape
    assert calls["init"]["flow_field_path"] == "dummy-flow-field.txt"
    assert calls["init"]["cache_steps"] == 0
    assert calls["run"] == dict(pairs=pairs, core_block_sites=256, flank_sites=64,
                                pair_batch_size=32, max_streams=3, mean_only=False,
                                return_posterior=False)


def test_infer_forwards_to_run_fb(monkeypatch, genotype_data):
    G, pos = genotype_data
    calls = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, calls=calls))
    r = gamma_smc_cu_b200.infer(G, pos, flow_field_path="ff.txt", return_posterior=True)
    n = G.shape[0]
    assert r["pairs"] == [(i, j) for i in range(n) for j in range(i)]
    assert calls["run_fb"]["return_posterior"] is True
    assert calls["run_fb"]["mean_only"] is True
    assert calls["init"]["Ne"] == 10000.0
    # auto theta: 4 Ne mu_eff equals the mean per-diploid heterozygosity
    het = (G[0::2] != G[1::2]).sum(axis=1).mean() / (pos[-1] + 1.0)
    np.testing.assert_allclose(4e4 * calls["init"]["mu"], het)
    np.testing.assert_allclose(calls["init"]["rho"] / calls["init"]["mu"], 0.8)
    r = gamma_smc_cu_b200.infer(G, pos, flow_field_path="ff.txt", auto_estimate_theta=False)
    assert (calls["init"]["mu"], calls["init"]["rho"]) == (1.25e-8, 1e-8)


def test_auto_core_block_sites_uses_recommendation(monkeypatch, genotype_data):
    G, pos = genotype_data
    captured = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "cuda_mem_info", lambda: (32 * 10**9, 40 * 10**9))
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, captured=captured))
    gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=[(0, 1), (2, 3)], flow_field_path="x",
                                      core_block_sites="auto", flank_sites=64)
    assert captured["core_block_sites"] == G.shape[1]
    assert captured["flank_sites"] == 64


def test_auto_core_block_sites_large_input(monkeypatch):
    """400k sites x 63,190 pairs on a 178 GB-free device picks the 32768 cap."""
    from gamma_smc_cu_b200.infer import _recommend_core_block_size
    core, est = _recommend_core_block_size(400_000, 63_190, True, 2048, 178 * 10**9)
    assert core == 32768
    assert est == 12 * (32768 + 4096) * 63_190


def test_warns_when_block_exceeds_memory(monkeypatch, genotype_data):
    G, pos = genotype_data
    monkeypatch.setattr(gamma_smc_cu_b200._core, "cuda_mem_info", lambda: (1024, 1024))
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos))
    with pytest.warns(UserWarning, match="GPU memory"):
        gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=[(0, 1)], flow_field_path="x",
                                          core_block_sites=8192, flank_sites=2048)


def test_auto_pair_batch_size_capped_by_n_pairs(monkeypatch, genotype_data):
    G, pos = genotype_data
    captured = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "cuda_mem_info", lambda: (32 * 10**9, 40 * 10**9))
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, captured=captured))
    pairs = [(0, 1), (2, 3), (4, 5)]
    gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=pairs, flow_field_path="x", pair_batch_size=-1)
    assert captured["pair_batch_size"] == len(pairs)


def test_auto_falls_back_when_query_fails(monkeypatch, genotype_data):
    G, pos = genotype_data

    def boom():
        raise RuntimeError("no cuda")

    monkeypatch.setattr(gamma_smc_cu_b200._core, "cuda_mem_info", boom)
    captured = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, captured=captured))
    with pytest.warns(UserWarning, match="could not query GPU"):
        gamma_smc_cu_b200.infer_blockwise(G, pos, pairs=[(0, 1)], flow_field_path="x",
                                          core_block_sites="auto")
    assert captured["core_block_sites"] == 8192


def test_segregating_filter_applied_before_context(monkeypatch, genotype_data):
    G, pos = genotype_data
    Gp = np.concatenate([np.zeros((G.shape[0], 1), np.uint8), G,
                         np.ones((G.shape[0], 1), np.uint8)], axis=1)
    pp = np.concatenate([[pos[0] - 1.0], pos, [pos[-1] + 1.0]])
    calls = {}
    monkeypatch.setattr(gamma_smc_cu_b200._core, "FlowContext", _fake_ctx(pos, calls=calls))
    r = gamma_smc_cu_b200.infer(Gp, pp, pairs=[(0, 1)], flow_field_path="x")
    assert calls["init"]["shape"] == G.shape
    np.testing.assert_array_equal(r["positions"], pos)


def test_default_flow_field_resolves():
    from gamma_smc_cu_b200.infer import _resolve_flow_field_path
    p = _resolve_flow_field_path(None)
    assert p.endswith("default_flow_field.txt")
    assert _resolve_flow_field_path("given.txt") == "given.txt"
