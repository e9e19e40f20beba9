"""Pins of the CPU oracle: reference-built tables, golden vectors, known answers.

These run without a GPU.  They establish that the oracle restates the
reference: its table builder is bit-identical to the reference's compiled
src/flow_field.cpp (when oracle/_ref was built from a reference checkout),
and its host logic reproduces the golden vectors the reference's own Python
made (tests/golden/make_host_golden.py).
"""
import hashlib
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _golden():
    with open(os.path.join(GOLDEN, "host_logic.json")) as f:
        return json.load(f)


def test_flow_field_fixture_sha(flow_field):
    want = open(os.path.join(GOLDEN, "flow_field.sha256")).read().split()[0]
    assert hashlib.sha256(open(flow_field, "rb").read()).hexdigest() == want


def test_flow_field_parses(oracle, flow_field):
    u, v, b = oracle.load_flow_field(flow_field)
    assert u.shape == (2550,) and v.shape == (2550,)
    assert np.isfinite(u).all() and np.isfinite(v).all()
    np.testing.assert_allclose(b, [-5.0, 2.0, -2.0, 0.0], atol=1e-6)


def test_flow_field_missing_file_raises(oracle):
    with pytest.raises(RuntimeError, match="Failed to load flow field"):
        oracle.load_flow_field("/nonexistent/flow_field.txt")


@pytest.mark.parametrize("Ne,mu,rho", [(1e4, 1.25e-8, 1e-8), (1e4, 2.9e-8, 2.3e-8),
                                       (5000.0, 1e-8, 1e-8), (2.5e4, 6e-9, 1.5e-8)])
def test_tables_bit_identical_to_reference_builder(oracle, flow_field, Ne, mu, rho):
    if oracle.ref_tables_lib() is None:
        pytest.skip("oracle/_ref/libref_tables.so not built (needs a reference checkout)")
    u, v, b = oracle.load_flow_field(flow_field)
    u2, v2, b2 = oracle.load_flow_field(flow_field, use_reference=True)
    assert np.array_equal(u, u2) and np.array_equal(v, v2) and np.array_equal(b, b2)
    ours = oracle.build_tables(u, v, b, 1000, Ne, mu, rho)
    ref = oracle.build_tables(u, v, b, 1000, Ne, mu, rho, use_reference=True)
    for k, name in enumerate(oracle.TABLE_NAMES):
        assert np.array_equal(ours[k], ref[k]), name


def test_tables_small_step_counts(oracle, flow_field):
    if oracle.ref_tables_lib() is None:
        pytest.skip("oracle/_ref/libref_tables.so not built")
    u, v, b = oracle.load_flow_field(flow_field)
    for L in (1, 2, 7):
        assert np.array_equal(oracle.build_tables(u, v, b, L, 1e4, 1.25e-8, 1e-8),
                              oracle.build_tables(u, v, b, L, 1e4, 1.25e-8, 1e-8,
                                                  use_reference=True))


def test_tables_finite_and_clamped(oracle, flow_field):
    T = oracle.tables_for(flow_field, 1e4, 1.25e-8, 1e-8)
    assert np.isfinite(T).all()
    # forward site tables are clipped to the grid
    for k in (4, 6):
        assert T[k].min() >= -5.0 and T[k].max() <= 2.0
    for k in (5, 7):
        assert T[k].min() >= -2.0 and T[k].max() <= 0.0


# --- golden vectors of the reference's host logic -------------------------

def test_theta_known_answers(oracle):
    """tests/unit/test_infer.py:98-144 restated."""
    G = np.array([[0, 0, 1, 1], [0, 1, 1, 1], [0, 0, 0, 1], [1, 0, 0, 1]], np.uint8)
    pos = np.array([10.0, 20.0, 30.0, 40.0])
    for est in (oracle.estimate_scaled_params, _pkg_theta()):
        mu_e, rho_e = est(G, pos, 2e-8, 5e-8, 1e4)
        np.testing.assert_allclose(4e4 * mu_e, 1.0 / 41.0)
        np.testing.assert_allclose(4e4 * rho_e, (1.0 / 41.0) * 2.5)
    G = np.array([[0, 1], [1, 1], [0, 0], [0, 1]], np.uint8)
    pos = np.array([100.0, 200.0])
    for est in (oracle.estimate_scaled_params, _pkg_theta()):
        mu_e, rho_e = est(G, pos, 2e-8, 5e-8, 1e4)
        np.testing.assert_allclose(4e4 * mu_e, 1.0 / 201.0)
        np.testing.assert_allclose(4e4 * rho_e, 2.5 / 201.0)


def _pkg_theta():
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    return _estimate_scaled_params


def test_theta_golden(oracle):
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    for case in _golden()["theta"]:
        G = np.array(case["G"], np.uint8).reshape(len(case["G"]), -1)
        pos = np.array(case["positions"], np.float64)
        for est in (oracle.estimate_scaled_params, _estimate_scaled_params):
            got = est(G, pos, case["mu"], case["rho"], case["Ne"])
            assert list(got) == case["expected"]


def test_filter_segregating_golden(oracle):
    from gamma_smc_cu_b200.infer import _filter_segregating
    for case in _golden()["segregating"]:
        G = np.array(case["G"], np.uint8)
        pos = np.arange(G.shape[1], dtype=np.float64) * 10.0
        for fn in (oracle.filter_segregating, _filter_segregating):
            Gf, pf, keep = fn(G, pos)
            assert keep.astype(int).tolist() == case["keep"]
            assert np.array_equal(Gf, G[:, keep]) and np.array_equal(pf, pos[keep])


def test_block_sizing_golden(oracle):
    import importlib
    I = importlib.import_module("gamma_smc_cu_b200.infer")
    g = _golden()
    for m in (True, False):
        assert I._gpu_bytes_per_pair_site(m) == g["bytes_per_pair_site"][str(m)]
    for c in g["sizing"]:
        for rec, est in ((oracle.recommend_core_block_size, oracle.estimate_block_gpu_bytes),
                         (I._recommend_core_block_size, I._estimate_block_gpu_bytes)):
            core, e = rec(c["n_sites"], c["n_pairs"], c["mean_only"], c["flank"], c["free"])
            assert (core, e) == (c["core"], c["est"]), c
            assert est(8192, c["flank"], c["n_pairs"], c["mean_only"],
                       n_sites=c["n_sites"]) == c["est_clamped"]


def test_block_windows_known_answers(oracle):
    """make_block_windows (src/bindings.cpp:2517-2534)."""
    w = oracle.make_block_windows(10, 4, 2)
    assert w.tolist() == [[0, 4, 0, 6], [4, 8, 2, 10], [8, 10, 6, 10]]
    assert oracle.make_block_windows(5, 5, 0).tolist() == [[0, 5, 0, 5]]
    assert oracle.make_block_windows(5, 100, 7).tolist() == [[0, 5, 0, 5]]
    assert oracle.make_block_windows(0, 8, 2).shape == (0, 4)


# --- bitpack and pair indexing (tests/unit/test_bitpack.py, test_pair_indexing.py)

@pytest.mark.parametrize("n,S,kind", [(10, 100, "rand"), (50, 1000, "zeros"), (50, 1000, "ones"),
                                      (4, 1, "rand"), (1, 500, "rand"), (10, 64, "rand"),
                                      (5, 128, "rand")])
def test_bitpack_roundtrip(oracle, n, S, kind):
    rng = np.random.RandomState(42 + S)
    G = {"rand": lambda: rng.randint(0, 2, size=(n, S)).astype(np.uint8),
         "zeros": lambda: np.zeros((n, S), np.uint8),
         "ones": lambda: np.ones((n, S), np.uint8)}[kind]()
    packed = oracle.bitpack(G)
    assert packed.shape == (n, (S + 63) // 64)
    assert np.array_equal(oracle.unpack(packed, n, S), G)
    # padding bits beyond S are zero
    if S % 64:
        assert int(packed[:, -1].max()) >> (S % 64) == 0


def test_pair_indexing_roundtrip(oracle):
    for n in (5, 10, 50):
        p = 0
        for i in range(1, n):
            for j in range(i):
                assert oracle.ij_to_pair(i, j) == p == oracle.ij_to_pair(j, i)
                assert oracle.pair_to_ij(p) == (i, j)
                p += 1
    for n in (2, 10, 100):
        assert oracle.ij_to_pair(n - 1, n - 2) == n * (n - 1) // 2 - 1


def test_default_pairs_are_row_major(oracle):
    from gamma_smc_cu_b200 import synthetic
    P = synthetic.all_pairs(12)
    assert [tuple(p) for p in P.tolist()] == oracle.all_pairs(12)
    assert [oracle.ij_to_pair(i, j) for i, j in P.tolist()] == list(range(len(P)))
    idx = np.arange(0, 20000, 7)
    assert all(oracle.ij_to_pair(int(i), int(j)) == int(k)
               for (i, j), k in zip(synthetic.pairs_from_index(idx), idx))


# --- scan invariants of the oracle (no GPU) -------------------------------

def test_oracle_scan_invariants(oracle, flow_field, small_data):
    G, pos = small_data
    pairs = [(1, 0), (2, 0), (39, 38), (20, 7)]
    r = oracle.infer(G, pos, pairs=pairs, flow_field_path=flow_field, mean_only=False,
                     return_posterior=True)
    m = r["mean"]
    assert m.shape == (G.shape[1], len(pairs)) and m.dtype == np.float32
    assert np.isfinite(m).all() and (m > 0).all()
    assert (r["lower"] <= m + 1e-3).all() and (m <= r["upper"] + 1e-3).all()
    recon = (r["posterior_alpha"] / r["posterior_beta"]) * 2.0 * 1e4
    np.testing.assert_allclose(recon, m, rtol=1e-4, atol=1e-2)
    base = oracle.infer(G, pos, pairs=pairs, flow_field_path=flow_field)
    assert np.array_equal(base["mean"], m)  # posterior flag does not change mean
    one = oracle.infer_blockwise(G, pos, pairs=pairs, flow_field_path=flow_field,
                                 core_block_sites=G.shape[1], flank_sites=0)
    assert np.array_equal(one["mean"], m)


def test_oracle_monomorphic_padding_invisible(oracle, flow_field, small_data):
    G, pos = small_data
    Gp = np.concatenate([np.zeros((G.shape[0], 1), np.uint8), G,
                         np.ones((G.shape[0], 1), np.uint8)], axis=1)
    pp = np.concatenate([[pos[0] - 1.0], pos, [pos[-1] + 1.0]])
    a = oracle.infer(G, pos, pairs=[(0, 1), (2, 3)], flow_field_path=flow_field)
    b = oracle.infer(Gp, pp, pairs=[(0, 1), (2, 3)], flow_field_path=flow_field)
    assert np.array_equal(a["mean"], b["mean"])
    assert np.array_equal(a["positions"], b["positions"])


def test_oracle_rejects_mismatched_positions(oracle, small_data):
    G, pos = small_data
    with pytest.raises(ValueError, match="positions length"):
        oracle.infer(G, pos[:-1], pairs=[(0, 1)], flow_field_path="x")


def test_bilinear_keeps_upper_boundary_cell(oracle):
    """tests/unit/test_gamma_smc_flow.py:140-158 on the scan's 51 x 50 grid:
    at the upper edge the interpolation keeps full weight on the last cell."""
    grid = (10.0 * np.arange(51)[:, None] + np.arange(50)[None, :]).astype(np.float32)
    assert oracle.layer_bilinear(grid, 2.0, 0.0) == pytest.approx(549.0)
    c_mid = -2.0 + 24 * (2.0 / 49)          # column 24 exactly
    assert oracle.layer_bilinear(grid, 2.0, c_mid) == pytest.approx(524.0, abs=1e-3)
    m_mid = -5.0 + 20 * 0.14                # row 20
    assert oracle.layer_bilinear(grid, m_mid, 0.0) == pytest.approx(249.0, abs=1e-3)
    # below the grid the lower cell is used
    assert oracle.layer_bilinear(grid, -9.0, -3.0) == pytest.approx(0.0)
