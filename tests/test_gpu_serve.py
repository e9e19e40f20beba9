"""The serving loop on the GPU: every query's result in the concurrent mix
equals the same query run alone through FlowContext.run_fb_window (the plain
per-call path), within the 1e-4 relative tolerance (bit-identical when no
window is chunked)."""
import threading
import time

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic
from gamma_smc_cu_b200.serve import TmrcaServer

pytestmark = pytest.mark.gpu

RTOL = 1e-4
NE = 1e4


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


def _mix(server, n_haps, S, clients=4, per_client=20, max_pairs=300, seed=0):
    allp = synthetic.all_pairs(n_haps)
    subs = []
    lock = threading.Lock()

    def client(k):
        rng = np.random.default_rng(seed + k)
        for q in range(per_client):
            n = int(rng.integers(1, min(max_pairs, len(allp)) + 1))
            pairs = allp[rng.choice(len(allp), n, replace=False)]
            w = int(np.exp(rng.uniform(0, np.log(S))))
            s0 = int(rng.integers(0, S - w + 1))
            mode = q % 5
            kw = dict(mean_only=mode != 1, return_posterior=mode == 2)
            f = server.submit(pairs, s0, s0 + w, **kw)
            with lock:
                subs.append((f, pairs, s0, s0 + w, kw))
            time.sleep(float(rng.exponential(0.002)))

    ts = [threading.Thread(target=client, args=(k,)) for k in range(clients)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return subs


def _check_alone(ctx, subs, exact):
    for f, pairs, s0, s1, kw in subs:
        got = f.result(timeout=120)
        want = ctx.run_fb_window(pairs, s0, s1, **kw)
        assert set(got) == set(want)
        for k in want:
            assert got[k].shape == want[k].shape
            assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))
            if exact:
                assert np.array_equal(got[k], want[k]), k


def test_served_results_equal_alone(small_data, oracle, flow_field):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    with TmrcaServer(ctx, positions=pos, max_inflight=3) as srv:
        subs = _mix(srv, G.shape[0], G.shape[1])
        f = srv.submit([(5, 2), (9, 0)], region_bp=(1e5, 3e5))
        s0, s1 = srv.sites_of(1e5, 3e5)
        subs.append((f, np.array([(5, 2), (9, 0)]), s0, s1, {}))
        _check_alone(ctx, subs, exact=True)
        st = srv.stats()
    assert st["completed"] == len(subs) and st.get("rejected", 0) == 0
    assert st["batches"] <= st["completed"]


@pytest.mark.parametrize("flank", [2048, 4])
def test_served_chunked_windows_exact(oracle, flow_field, flank):
    """Chunked windows in the served mix equal the query decoded alone bit for
    bit; a 4-site burn-in makes chunks fail the device check and the server
    redo those queries whole."""
    G, pos = synthetic.cohort("chrom", n_sites=12000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    with TmrcaServer(ctx, positions=pos, max_inflight=2, core_block_sites=2048,
                     flank_sites=flank, tile_width=32) as srv:
        subs = _mix(srv, G.shape[0], G.shape[1], clients=2, per_client=10, max_pairs=200)
        _check_alone(ctx, subs, exact=True)
        st = srv.stats()
    if flank == 4:
        assert st.get("redone_whole", 0) > 0


def test_server_rejects_query_beyond_budget(small_data, oracle, flow_field):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    with TmrcaServer(ctx, positions=pos, max_inflight=1, hbm_budget=1 << 20) as srv:
        big = srv.submit(synthetic.all_pairs(40), 0, G.shape[1])   # 6.6 MB of means
        small = srv.submit([(1, 0)], 0, 100)
        with pytest.raises(MemoryError):
            big.result(timeout=60)
        assert small.result(timeout=60)["mean"].shape == (100, 1)
