"""Multi-device pair sharding without a GPU.

The per-device contexts are stood in for by the oracle (each decodes its
shard on the CPU), so what is checked is the host logic: the reference's pair
split (python/gamma_smc_cu/multigpu.py:59-70), the concatenation of per-part
results along the pair axis, the pair-weighted summary merge
(multigpu.py:73-103), and -- for the one-process-per-GPU form -- a
world-size-2 ``gloo`` group whose gathered results and all-reduced summaries
must equal one process decoding every pair.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from gamma_smc_cu_b200.multigpu import (DistributedFlowContext, MultiGPUFlowContext,
                                        split_pairs)


class OracleContext:
    """FlowContext stand-in: the same methods, answered by the oracle."""

    def __init__(self, G, positions, Ne, mu, rho, flow_field_path, cache_steps):
        self.args = (G, positions)
        self.params = (Ne, mu, rho, flow_field_path)
        self.calls = []

    def run_fb(self, pairs, mean_only=True, return_posterior=False):
        from oracle import oracle as O
        self.calls.append(("run_fb", len(pairs)))
        return O.run_fb(*self.args, [tuple(p) for p in pairs], *self.params, mean_only,
                        return_posterior)

    def run_fwd(self, pairs, mean_only=True):
        from oracle import oracle as O
        self.calls.append(("run_fwd", len(pairs)))
        return O.run_fwd(*self.args, [tuple(p) for p in pairs], *self.params, mean_only)

    def run_fb_summary(self, pairs):
        from oracle import oracle as O
        self.calls.append(("run_fb_summary", len(pairs)))
        return O.run_fb_summary(*self.args, [tuple(p) for p in pairs], *self.params)


@pytest.fixture(scope="module")
def setup(flow_field):
    from gamma_smc_cu_b200 import synthetic
    from oracle import oracle as O
    pos = synthetic.positions_for(300, 2.0e5, 11)
    G = synthetic.haplotypes(12, pos, 12)
    mu, rho = O.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    pairs = [tuple(p) for p in synthetic.all_pairs(G.shape[0])]
    return G, pos, 1e4, mu, rho, flow_field, pairs


def test_split_pairs_matches_reference_rule():
    assert split_pairs(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert split_pairs(5, 4) == [(0, 2), (2, 4), (4, 5), (5, 5)]
    assert split_pairs(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    assert split_pairs(0, 2) == [(0, 0), (0, 0)]
    for n in range(0, 40):
        for k in range(1, 9):
            parts = split_pairs(n, k)
            assert len(parts) == k and parts[0][0] == 0 and parts[-1][1] == n
            assert all(a <= b for a, b in parts)
            assert all(parts[i][1] == parts[i + 1][0] for i in range(k - 1))


def test_multi_context_run_fb_concatenates_shards(setup):
    from oracle import oracle as O
    G, pos, Ne, mu, rho, ff, pairs = setup
    m = MultiGPUFlowContext(G, pos, Ne, mu, rho, ff, gpu_ids=[0, 1, 2],
                            context_factory=OracleContext)
    try:
        got = m.run_fb(pairs, mean_only=False)
        want = O.run_fb(G, pos, pairs, Ne, mu, rho, ff, False, False)
        assert set(got) == {"mean", "lower", "upper"}
        for k in got:
            assert got[k].shape == (G.shape[1], len(pairs))
            np.testing.assert_array_equal(got[k], want[k])
        # every device got its ceil(n/3) share
        sizes = [c.calls[-1][1] for c in m.contexts]
        assert sizes == [b - a for a, b in split_pairs(len(pairs), 3)]
        assert m.device_ids == [0, 1, 2]
    finally:
        m.close()


def test_multi_context_run_fwd_and_idle_devices(setup):
    from oracle import oracle as O
    G, pos, Ne, mu, rho, ff, pairs = setup
    m = MultiGPUFlowContext(G, pos, Ne, mu, rho, ff, gpu_ids=[0, 1, 2, 3],
                            context_factory=OracleContext)
    try:
        few = pairs[:3]  # the fourth device gets nothing
        got = m.run_fwd(few)
        want = O.run_fwd(G, pos, few, Ne, mu, rho, ff, True)
        np.testing.assert_array_equal(got["mean"], want["mean"])
        assert m.contexts[3].calls == []
    finally:
        m.close()


def test_multi_context_empty_pairs(setup):
    G, pos, Ne, mu, rho, ff, _ = setup
    m = MultiGPUFlowContext(G, pos, Ne, mu, rho, ff, gpu_ids=[0, 1],
                            context_factory=OracleContext)
    try:
        r = m.run_fb([], mean_only=False)
        assert {k: v.shape for k, v in r.items()} == {
            "mean": (G.shape[1], 0), "lower": (G.shape[1], 0), "upper": (G.shape[1], 0)}
        assert m.run_fwd([])["mean"].shape == (G.shape[1], 0)
        s = m.run_fb_summary([])
        assert s["n_pairs"] == 0 and s["n_gpus"] == 0
        np.testing.assert_array_equal(s["site_mean"], np.zeros(G.shape[1], np.float32))
    finally:
        m.close()


def test_multi_context_summary_merges_chunks(setup):
    from oracle import oracle as O
    G, pos, Ne, mu, rho, ff, pairs = setup
    m = MultiGPUFlowContext(G, pos, Ne, mu, rho, ff, gpu_ids=[0, 1],
                            context_factory=OracleContext)
    try:
        got = m.run_fb_summary(pairs, chunk_size=7)
        full = O.run_fb(G, pos, pairs, Ne, mu, rho, ff, True, False)["mean"]
        assert got["n_pairs"] == len(pairs) and got["n_gpus"] == 2
        # float32 chunk means re-weighted in float64: a few float32 ulps
        np.testing.assert_allclose(got["site_mean"], full.astype(np.float64).mean(axis=1),
                                   rtol=1e-6)
        np.testing.assert_array_equal(got["site_min"], full.min(axis=1))
        np.testing.assert_array_equal(got["site_max"], full.max(axis=1))
        # chunks of at most 7 pairs on each device
        assert all(n <= 7 for c in m.contexts for _, n in c.calls)
    finally:
        m.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dist_worker(rank, world, port, setup, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        G, pos, Ne, mu, rho, ff, pairs = setup
        d = DistributedFlowContext(G, pos, Ne, mu, rho, ff, context_factory=OracleContext)
        full = d.run_fb(pairs, mean_only=False)
        shard = d.run_fb(pairs, gather=False)
        fwd = d.run_fwd(pairs[:5])
        summ = d.run_fb_summary(pairs, chunk_size=9)
        out = {"shard_mean": shard["mean"], "summ_mean": summ["site_mean"],
               "summ_min": summ["site_min"], "summ_max": summ["site_max"],
               "summ_n": summ["n_pairs"], "shard": np.array(d.shard(len(pairs)))}
        if rank == 0:
            out.update({"full_" + k: v for k, v in full.items()})
            out["fwd_mean"] = fwd["mean"]
        else:
            out["full_is_none"] = full is None and fwd is None
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **out)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_distributed_two_ranks_gloo(setup, tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    G, pos, Ne, mu, rho, ff, pairs = setup
    world = 2
    mp.start_processes(_dist_worker, args=(world, _free_port(), setup, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    want = O.run_fb(G, pos, pairs, Ne, mu, rho, ff, False, False)
    for k in ("mean", "lower", "upper"):
        np.testing.assert_array_equal(r0["full_" + k], want[k])
    assert bool(r1["full_is_none"])
    np.testing.assert_array_equal(
        r0["fwd_mean"], O.run_fwd(G, pos, pairs[:5], Ne, mu, rho, ff, True)["mean"])
    # shards are the reference split and cover the pairs in order
    (a0, b0), (a1, b1) = split_pairs(len(pairs), world)
    assert tuple(r0["shard"]) == (a0, b0) and tuple(r1["shard"]) == (a1, b1)
    np.testing.assert_array_equal(r0["shard_mean"], want["mean"][:, a0:b0])
    np.testing.assert_array_equal(r1["shard_mean"], want["mean"][:, a1:b1])
    # the all-reduced summary is identical on both ranks and matches one process
    for k in ("summ_mean", "summ_min", "summ_max"):
        np.testing.assert_array_equal(r0[k], r1[k])
    assert int(r0["summ_n"]) == len(pairs)
    np.testing.assert_allclose(r0["summ_mean"],
                               want["mean"].astype(np.float64).mean(axis=1), rtol=1e-6)
    np.testing.assert_array_equal(r0["summ_min"], want["mean"].min(axis=1))
    np.testing.assert_array_equal(r0["summ_max"], want["mean"].max(axis=1))
