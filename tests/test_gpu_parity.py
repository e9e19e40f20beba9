"""Parity of the CUDA path with the oracle (and with the reference's compiled
code when oracle/_ref holds it), through the C ABI.

Tolerance: 1e-4 relative on the posterior mean is the bar for this path; the
kernels are written to be bit-identical, which the *_bit_exact tests check.
"""
import ctypes
import importlib.util

import numpy as np
import pytest

import gamma_smc_cu_b200 as G200
from gamma_smc_cu_b200 import _core, _lib, synthetic

pytestmark = pytest.mark.gpu

RTOL = 1e-4
NE = 1e4
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


def _assert_parity(got, want, keys=KEYS, exact=True):
    for k in keys:
        if k not in want:
            assert k not in got, k
            continue
        assert got[k].shape == want[k].shape and got[k].dtype == np.float32, k
        assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))
        if exact:
            assert np.array_equal(got[k], want[k]), (k, _max_rel(got[k], want[k]))


@pytest.fixture(scope="module")
def small(small_data, oracle, flow_field):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    return G, pos, mu, rho


def test_tables_match_oracle_bit_exact(small, oracle, flow_field):
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    T = oracle.tables_for(flow_field, NE, mu, rho)
    # scan table t -> oracle (mean, cv) table indices
    src = {0: (4, 5), 1: (6, 7), 2: (8, 9), 3: (10, 11)}
    for t, (im, ic) in src.items():
        for layer in (0, 1, 2, 17, 499, 998, 999):
            m, c = ctx.table_layer(t, layer)
            assert np.array_equal(m.ravel(), T[im, layer]), (t, layer)
            assert np.array_equal(c.ravel(), T[ic, layer]), (t, layer)
    m, c = ctx.table_layer(4, 0)
    assert np.array_equal(m.ravel(), T[2, 999]) and np.array_equal(c.ravel(), T[3, 999])


def test_infer_full_posterior_bit_exact(small, oracle, flow_field):
    G, pos, _, _ = small
    want = oracle.infer(G, pos, flow_field_path=flow_field, mean_only=False,
                        return_posterior=True)
    got = G200.infer(G, pos, flow_field_path=flow_field, mean_only=False, return_posterior=True)
    assert got["pairs"] == want["pairs"] and len(got["pairs"]) == 780
    np.testing.assert_array_equal(got["positions"], want["positions"])
    _assert_parity(got, want)


def test_infer_mean_only_and_flags(small, oracle, flow_field):
    G, pos, _, _ = small
    pairs = [(1, 0), (5, 3), (39, 2), (17, 16)]
    want = oracle.infer(G, pos, pairs=pairs, flow_field_path=flow_field)
    got = G200.infer(G, pos, pairs=pairs, flow_field_path=flow_field)
    assert set(got) == {"mean", "pairs", "positions"}
    _assert_parity(got, want)
    post = G200.infer(G, pos, pairs=pairs, flow_field_path=flow_field, return_posterior=True)
    assert np.array_equal(post["mean"], got["mean"])
    recon = (post["posterior_alpha"] / post["posterior_beta"]) * 2.0 * NE
    np.testing.assert_allclose(recon, post["mean"], rtol=1e-4, atol=1e-2)
    ci = G200.infer(G, pos, pairs=pairs, flow_field_path=flow_field, mean_only=False)
    assert (ci["lower"] <= ci["mean"] + 1e-3).all() and (ci["mean"] <= ci["upper"] + 1e-3).all()
    assert (got["mean"] > 0).all()


@pytest.mark.parametrize("core,flank", [(300, 100), (64, 17), (1000, 2048), (129, 1),
                                        (2127, 0), (5000, 0), (1, 3)])
def test_blockwise_matches_oracle(small, oracle, flow_field, core, flank):
    G, pos, _, _ = small
    pairs = [(i, j) for i in range(0, 40, 3) for j in range(i)][:150]
    want = oracle.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                                  core_block_sites=core, flank_sites=flank, mean_only=False,
                                  return_posterior=True)
    got = G200.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                               core_block_sites=core, flank_sites=flank, mean_only=False,
                               return_posterior=True)
    np.testing.assert_array_equal(got["blocks"], want["blocks"])
    _assert_parity(got, want)


def test_blockwise_single_block_equals_infer(small, flow_field):
    G, pos, _, _ = small
    pairs = [(0, 1), (2, 3)]
    full = G200.infer(G, pos, pairs=pairs, flow_field_path=flow_field)
    blk = G200.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                               core_block_sites=G.shape[1], flank_sites=0, pair_batch_size=1)
    np.testing.assert_allclose(blk["mean"], full["mean"], rtol=1e-5, atol=1e-6)
    assert np.array_equal(blk["mean"], full["mean"])
    np.testing.assert_array_equal(blk["blocks"], [[0, G.shape[1], 0, G.shape[1]]])


def test_pair_chunking_and_streams_do_not_change_values(small, flow_field):
    G, pos, _, _ = small
    pairs = [(i, j) for i in range(40) for j in range(i)]
    kw = dict(pairs=pairs, flow_field_path=flow_field, core_block_sites=500, flank_sites=200)
    a = G200.infer_blockwise(G, pos, **kw)
    b = G200.infer_blockwise(G, pos, pair_batch_size=7, **kw)
    c = G200.infer_blockwise(G, pos, max_streams=2, **kw)
    assert np.array_equal(a["mean"], b["mean"]) and np.array_equal(a["mean"], c["mean"])


def test_edge_positions_and_shapes(oracle, flow_field):
    """Gaps beyond the 1000-step cache, zero and half-bp gaps, site 0 at 0,
    S = 1, and windows that start inside a 64/128-site word."""
    rng = np.random.default_rng(11)
    gaps = np.array([0.0, 1.0, 0.5, 1.5, 2.5, 999, 1000, 1001, 1999, 2000, 2001, 15000,
                     250000, 3, 0.0, 7] * 20)
    pos = np.cumsum(gaps)
    S = len(pos)
    G = (rng.random((12, S)) < 0.3).astype(np.uint8)
    G[0, :] = 1 - G[1, :]  # force segregating everywhere
    pairs = [(1, 0), (5, 2), (11, 3), (4, 4)]
    for core, flank in ((S, 0), (37, 11), (128, 64), (200, 0) if S <= 200 else (S, 0)):
        want = oracle.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                                      core_block_sites=core, flank_sites=flank,
                                      mean_only=False, return_posterior=True)
        got = G200.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                                   core_block_sites=core, flank_sites=flank, mean_only=False,
                                   return_posterior=True)
        _assert_parity(got, want)
    # a single site
    G1 = np.array([[0], [1], [1], [0]], np.uint8)
    p1 = np.array([12345.0])
    want = oracle.infer(G1, p1, pairs=[(1, 0), (3, 0)], flow_field_path=flow_field,
                        mean_only=False, return_posterior=True)
    got = G200.infer(G1, p1, pairs=[(1, 0), (3, 0)], flow_field_path=flow_field,
                     mean_only=False, return_posterior=True)
    _assert_parity(got, want)


def test_empty_pairs_and_errors(small, flow_field):
    G, pos, _, _ = small
    r = G200.infer(G, pos, pairs=[], flow_field_path=flow_field)
    assert r["mean"].shape == (G.shape[1], 0)
    r = G200.infer_blockwise(G, pos, pairs=[], flow_field_path=flow_field, return_posterior=True,
                             core_block_sites=100, flank_sites=10)
    assert r["mean"].shape == (G.shape[1], 0) and r["posterior_alpha"].shape == (G.shape[1], 0)
    assert r["blocks"].shape == (22, 4)
    with pytest.raises(ValueError, match="out of range"):
        G200.infer(G, pos, pairs=[(0, 40)], flow_field_path=flow_field)
    with pytest.raises(RuntimeError, match="Failed to load flow field"):
        G200.infer(G, pos, pairs=[(0, 1)], flow_field_path="/nonexistent/ff.txt")


def test_context_properties_and_mem_info(small, flow_field):
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    assert (ctx.n_haps, ctx.n_sites) == G.shape
    assert ctx.device_id == _core.get_device()
    free, total = _core.cuda_mem_info()
    assert 0 < free <= total
    assert _core.get_device_count() >= 1


def test_bitpack_roundtrip_device(oracle):
    rng = np.random.RandomState(3)
    for n, S in ((10, 100), (4, 1), (1, 500), (10, 64), (5, 128), (33, 1000)):
        G = rng.randint(0, 2, size=(n, S)).astype(np.uint8)
        packed = _core.bitpack(G)
        assert np.array_equal(packed, oracle.bitpack(G))
        assert np.array_equal(_core.unpack(packed, n, S), G)
    for G in (np.zeros((50, 1000), np.uint8), np.ones((50, 1000), np.uint8)):
        assert np.array_equal(_core.unpack(_core.bitpack(G), 50, 1000), G)


def test_device_entry_point_matches_host(small, flow_field):
    import torch
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = np.array([(i, j) for i in range(40) for j in range(i)], np.int32)
    host = ctx.run_fb_blockwise([tuple(p) for p in pairs], core_block_sites=700, flank_sites=300,
                                pair_batch_size=-1, mean_only=False, return_posterior=True)
    dev = torch.device("cuda", ctx.device_id)
    P = len(pairs)
    pad = 5
    pi = torch.from_numpy(pairs[:, 0].copy()).to(dev)
    pj = torch.from_numpy(pairs[:, 1].copy()).to(dev)
    outs = [torch.full((G.shape[1], P + pad), -1.0, device=dev) for _ in range(5)]
    _lib.check(_lib.load().gsmc_run_fb_blockwise_device(
        ctx.handle, pi.data_ptr(), pj.data_ptr(), P, 700, 300, _lib.GSMC_CI | _lib.GSMC_POSTERIOR,
        *[o.data_ptr() for o in outs], P + pad, pad, None))
    torch.cuda.synchronize()
    for k, o in zip(KEYS, outs):
        o = o.cpu().numpy()
        assert np.array_equal(o[:, pad:], host[k]), k
        assert (o[:, :pad] == -1.0).all()


def test_oracle_and_cuda_match_reference_gpu_build(small, oracle, flow_field, ref_core):
    """The reference's own _core (compiled from its sources for sm_100a into
    oracle/_ref) on the same inputs: pins the oracle's scan restatement."""
    ref = ref_core
    if ref is None:
        pytest.skip("reference _core not built in oracle/_ref")
    G, pos, mu, rho = small
    pairs = [(i, j) for i in range(40) for j in range(i)]
    rctx = ref.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    want = rctx.run_fb(pairs, mean_only=False, return_posterior=True)
    orc = oracle.run_fb(G, pos, pairs, NE, mu, rho, flow_field, mean_only=False,
                        return_posterior=True)
    _assert_parity(orc, want)
    ours = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fb(
        pairs, mean_only=False, return_posterior=True)
    _assert_parity(ours, want)
    wantb = rctx.run_fb_blockwise(pairs[:100], core_block_sites=400, flank_sites=150,
                                  pair_batch_size=64, max_streams=1, mean_only=False,
                                  return_posterior=True)
    oursb = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fb_blockwise(
        pairs[:100], core_block_sites=400, flank_sites=150, pair_batch_size=64,
        max_streams=1, mean_only=False, return_posterior=True)
    np.testing.assert_array_equal(oursb["blocks"], wantb["blocks"])
    _assert_parity(oursb, wantb)


def test_chromosome_shape_sampled_pairs(oracle, flow_field):
    """356 haplotypes x 20k sites, 4096 pairs on the GPU; 48 sampled pairs
    checked against the oracle, the rest through size-independent properties."""
    G, pos = synthetic.cohort("chrom", n_sites=20000)
    pairs = synthetic.random_pairs(356, 4096, 9)
    got = G200.infer_blockwise(G, pos, pairs=pairs, core_block_sites=8192, flank_sites=2048,
                               mean_only=False, return_posterior=True)
    m = got["mean"]
    assert m.shape == (20000, 4096) and np.isfinite(m).all() and (m > 0).all()
    assert (got["lower"] <= m + 1e-3).all() and (m <= got["upper"] + 1e-3).all()
    sel = np.random.default_rng(1).choice(4096, 48, replace=False)
    want = oracle.infer_blockwise(G, pos, pairs=pairs[sel], core_block_sites=8192,
                                  flank_sites=2048, flow_field_path=flow_field, mean_only=False,
                                  return_posterior=True)
    for k in KEYS:
        assert np.array_equal(got[k][:, sel], want[k]), k


def test_gpu_calibration_counts_match_host(oracle):
    """The per-diploid het counts infer() makes on the GPU equal the host
    counts exactly, so the calibrated rates are identical."""
    from gamma_smc_cu_b200.infer import _estimate_scaled_params, _scaled_rates
    for name, S in (("small", None), ("chrom", 30000)):
        G, pos = synthetic.cohort(name, n_sites=S)
        got = _core.diploid_het_counts(G)
        assert got.dtype == np.int64 and np.array_equal(got, oracle.diploid_het_counts(G))
        assert _scaled_rates(G, pos, 1.25e-8, 1e-8, NE, True) == \
            _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    G = (np.random.default_rng(3).random((7, 333)) < 0.5).astype(np.uint8)  # odd n, ragged S
    assert np.array_equal(_core.diploid_het_counts(G), oracle.diploid_het_counts(G))
    assert _core.diploid_het_counts(np.zeros((6, 0), np.uint8)).tolist() == [0, 0, 0]


def test_two_pairs_per_thread_on_large_calls(oracle, flow_field):
    """A call with enough pair tiles to give every resident CTA two tasks runs
    two pairs per thread; a small one runs one.  Both stay bit-exact."""
    pos = synthetic.positions_for(20000, 4.0e6, 71)
    G = synthetic.haplotypes(64, pos, 72)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = [tuple(p) for p in synthetic.all_pairs(G.shape[0])]      # 2,016 pairs
    got = ctx.run_fb_blockwise(pairs, core_block_sites=64, flank_sites=32,
                               pair_batch_size=len(pairs))           # 313 windows x 8 tiles
    assert ctx.scan_shape() == (128, 2)
    want = oracle.run_fb_blockwise(G, pos, pairs, NE, mu, rho, flow_field, 64, 32)
    np.testing.assert_array_equal(got["mean"], want["mean"])
    few = pairs[:40]
    got = ctx.run_fb_blockwise(few, core_block_sites=4096, flank_sites=512,
                               pair_batch_size=len(few))
    assert ctx.scan_shape() == (128, 1)
    want = oracle.run_fb_blockwise(G, pos, few, NE, mu, rho, flow_field, 4096, 512)
    np.testing.assert_array_equal(got["mean"], want["mean"])


def test_release_scratch_then_rerun(small, flow_field):
    G, pos, mu, rho = small
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    pairs = [(i, j) for i in range(30) for j in range(i)]
    first = ctx.run_fb_blockwise(pairs, core_block_sites=300, flank_sites=100)["mean"]
    v = ctypes.c_uint64()
    _lib.check(_lib.load().gsmc_ctx_scratch_bytes(ctx.handle, ctypes.byref(v)))
    before = v.value
    ctx.release_scratch()
    _lib.check(_lib.load().gsmc_ctx_scratch_bytes(ctx.handle, ctypes.byref(v)))
    pool_free = v.value  # only the pair-index buffer is kept
    assert pool_free < before
    again = ctx.run_fb_blockwise(pairs, core_block_sites=300, flank_sites=100)["mean"]
    np.testing.assert_array_equal(first, again)
    ctx.release_scratch()
    ctx.release_scratch()  # idempotent
    _lib.check(_lib.load().gsmc_ctx_scratch_bytes(ctx.handle, ctypes.byref(v)))
    assert v.value == pool_free
