"""Scan-table sets on the GPU: several parameter sets alive at once, built
concurrently, reused after their last context closes, and the optional
float64 GPU build.

The reference keeps one process-global table set and frees it when a context
with other (Ne, mu, rho) is made, although earlier contexts still point into
it (src/bindings.cpp:2025-2041, 2649-2655).  Here every parameter set has its
own resident tables; these tests interleave calls on two live contexts with
different parameters and check each against the oracle bit for bit.
"""
import threading

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic

pytestmark = pytest.mark.gpu

PARAMS = ((1e4, 1.25e-8, 1e-8), (2e4, 2.0e-8, 0.5e-8), (5e3, 1.0e-8, 3e-8))
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


@pytest.fixture(scope="module")
def data(oracle, flow_field):
    G, pos = synthetic.cohort("small")
    pairs = [(i, j) for i in range(20) for j in range(i)]
    want = [oracle.run_fb(G, pos, pairs, ne, mu, rho, flow_field, mean_only=False,
                          return_posterior=True) for ne, mu, rho in PARAMS]
    return G, pos, pairs, want


def _same(got, want):
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k


def test_two_live_contexts_with_different_parameters(data, flow_field):
    G, pos, pairs, want = data
    a = _core.FlowContext(G, pos, *PARAMS[0], flow_field, 0)
    b = _core.FlowContext(G, pos, *PARAMS[1], flow_field, 0)
    for _ in range(2):   # interleaved calls on both
        _same(a.run_fb(pairs, mean_only=False, return_posterior=True), want[0])
        _same(b.run_fb(pairs, mean_only=False, return_posterior=True), want[1])
    b.close()            # a's tables stay valid after b goes
    _same(a.run_fb(pairs, mean_only=False, return_posterior=True), want[0])
    a.close()


def test_concurrent_creation_and_parked_reuse(data, flow_field):
    G, pos, pairs, want = data
    _core.free_cached_tables()
    ctxs = [None] * 6
    errors = []

    def make(i):
        try:
            ctxs[i] = _core.FlowContext(G, pos, *PARAMS[i % 3], flow_field, 0)
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=make, args=(i,)) for i in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    infos = [c.tables_info() for c in ctxs]
    # each parameter set was built exactly once, the other context reused it
    for p in range(3):
        built = [i for i in range(6) if i % 3 == p and not infos[i]["reused"]]
        assert len(built) == 1
        assert infos[built[0]]["build_seconds"] > 0
    for i, c in enumerate(ctxs):
        _same(c.run_fb(pairs, mean_only=False, return_posterior=True), want[i % 3])
    for c in ctxs:
        c.close()
    # the last set released stays resident for the next context with it
    last = 5 % 3   # contexts closed in order: the last one released holds PARAMS[2]
    again = _core.FlowContext(G, pos, *PARAMS[last], flow_field, 0)
    assert again.tables_info() == {"build_seconds": 0.0, "reused": True}
    _same(again.run_fb(pairs, mean_only=False, return_posterior=True), want[last])
    again.close()
    _core.free_cached_tables()
    fresh = _core.FlowContext(G, pos, *PARAMS[last], flow_field, 0)
    assert not fresh.tables_info()["reused"]
    _same(fresh.run_fb(pairs, mean_only=False, return_posterior=True), want[last])
    fresh.close()


def test_failed_build_reports_and_recovers(data, flow_field, tmp_path):
    G, pos, pairs, want = data
    with pytest.raises(RuntimeError, match="flow field"):
        _core.FlowContext(G, pos, *PARAMS[0], str(tmp_path / "missing.txt"), 0)
    c = _core.FlowContext(G, pos, *PARAMS[0], flow_field, 0)
    _same(c.run_fb(pairs, mean_only=False, return_posterior=True), want[0])
    c.close()


def test_gpu_float64_tables(data, flow_field):
    """The optional float64 GPU table build: a resident set of its own, tables
    within float32 rounding noise of the bit-exact host build's, posterior
    means close to the host tables' (the deviation is reported; the host
    build stays the parity default)."""
    G, pos, pairs, want = data
    a = _core.FlowContext(G, pos, *PARAMS[0], flow_field, 0)
    b = _core.FlowContext(G, pos, *PARAMS[0], flow_field, 0, table_build="gpu_fp64")
    assert not b.tables_info()["reused"]          # not the float32 set
    for t in range(5):
        for layer in ((0, 1, 17, 999) if t < 4 else (0,)):
            (m32, c32), (m64, c64) = a.table_layer(t, layer), b.table_layer(t, layer)
            assert np.isfinite(m64).all() and np.isfinite(c64).all()
            assert np.max(np.abs(m64 - m32)) < 2e-2 and np.max(np.abs(c64 - c32)) < 2e-2, (t, layer)
    r32 = a.run_fb(pairs, mean_only=False, return_posterior=True)
    _same(r32, want[0])
    r64 = b.run_fb(pairs, mean_only=False, return_posterior=True)
    rel = np.max(np.abs(r64["mean"].astype(np.float64) - r32["mean"]) / r32["mean"])
    print(f"float64 tables: max rel posterior-mean deviation {rel:.3e}")
    assert np.isfinite(r64["mean"]).all() and rel < 5e-2
    with pytest.raises(ValueError, match="table_build"):
        _core.FlowContext(G, pos, *PARAMS[0], flow_field, 0, table_build="fp16")
    a.close()
    b.close()
