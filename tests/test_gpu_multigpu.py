"""MultiGPUFlowContext on the GPU: its shards decoded by real contexts must
join into exactly the single-context result.

Only one device is visible to these tests, so the "devices" are several
contexts on device 0 driven concurrently by the pool's threads; the split,
concatenation and summary merge are the same code a multi-device run uses.
Per-pair outputs are bit-exact (pairs are independent); the merged site_mean
is a float64 pair-weighted sum of float32 chunk means, 1e-6 relative.
"""
import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic
from gamma_smc_cu_b200.multigpu import MultiGPUFlowContext

pytestmark = pytest.mark.gpu

NE = 1e4


@pytest.fixture(scope="module")
def small(small_data, oracle):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    return G, pos, mu, rho


def test_multi_context_matches_single(small, flow_field, oracle):
    G, pos, mu, rho = small
    pairs = [tuple(p) for p in synthetic.all_pairs(G.shape[0])]
    single = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    m = MultiGPUFlowContext(G, pos, NE, mu, rho, flow_field, gpu_ids=[0, 0, 0])
    try:
        got = m.run_fb(pairs, mean_only=False)
        want = single.run_fb(pairs, mean_only=False)
        for k in ("mean", "lower", "upper"):
            np.testing.assert_array_equal(got[k], want[k])
        np.testing.assert_array_equal(got["mean"], oracle.run_fb(
            G, pos, pairs, NE, mu, rho, flow_field, True, False)["mean"])
        fwd = m.run_fwd(pairs[:40])
        np.testing.assert_array_equal(fwd["mean"], single.run_fwd(pairs[:40])["mean"])
        s = m.run_fb_summary(pairs, chunk_size=25)
        full = want["mean"].astype(np.float64)
        assert s["n_pairs"] == len(pairs) and s["n_gpus"] == 3
        np.testing.assert_allclose(s["site_mean"], full.mean(axis=1), rtol=1e-6)
        np.testing.assert_array_equal(s["site_min"], want["mean"].min(axis=1))
        np.testing.assert_array_equal(s["site_max"], want["mean"].max(axis=1))
    finally:
        m.close()
        single.close()


def test_distributed_context_single_rank_nccl(small, flow_field, oracle):
    """The one-process-per-GPU form over a real NCCL group (one rank here):
    the gathered run_fb and the all-reduced summary on CUDA tensors equal
    one context's results."""
    import socket
    from datetime import timedelta

    import torch.distributed as dist
    from gamma_smc_cu_b200.multigpu import DistributedFlowContext
    G, pos, mu, rho = small
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        pairs = [tuple(p) for p in synthetic.all_pairs(G.shape[0])]
        d = DistributedFlowContext(G, pos, NE, mu, rho, flow_field)
        got = d.run_fb(pairs, mean_only=False)
        want = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0).run_fb(pairs, mean_only=False)
        for k in ("mean", "lower", "upper"):
            np.testing.assert_array_equal(got[k], want[k])
        s = d.run_fb_summary(pairs, chunk_size=300)
        full = want["mean"].astype(np.float64)
        assert s["n_pairs"] == len(pairs) and s["n_gpus"] == 1
        np.testing.assert_allclose(s["site_mean"], full.mean(axis=1), rtol=1e-6)
        np.testing.assert_array_equal(s["site_min"], want["mean"].min(axis=1))
        np.testing.assert_array_equal(s["site_max"], want["mean"].max(axis=1))
        d.close()
    finally:
        dist.destroy_process_group()
