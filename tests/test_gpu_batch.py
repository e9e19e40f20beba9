"""Batched jobs and per-window queries on the GPU against the oracle.

A job (pairs x site window) is decoded as one padded window of the
reference's block kernels (src/kernels/gamma_smc_flow.cu:632-669, 762-839);
the oracle's fb_window restates exactly that.  Tolerance: 1e-4 relative on
every output, and bit-identical where the kernels are (all of these checks:
chunked jobs are verified on the device and redone whole when their chunks
did not join).
"""
import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, synthetic
from gamma_smc_cu_b200.batch import Executor, Job, run_jobs

pytestmark = pytest.mark.gpu

RTOL = 1e-4
NE = 1e4
KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


def _check(got, want, exact=True):
    for k in KEYS:
        if k not in want:
            assert k not in got, k
            continue
        assert got[k].shape == want[k].shape, (k, got[k].shape, want[k].shape)
        assert _max_rel(got[k], want[k]) <= RTOL, (k, _max_rel(got[k], want[k]))
        if exact:
            assert np.array_equal(got[k], want[k]), (k, _max_rel(got[k], want[k]))


@pytest.fixture(scope="module")
def small_ctx(small_data, oracle, flow_field):
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    tables = oracle.tables_for(flow_field, NE, mu, rho)
    return ctx, G, pos, oracle.bitpack(G), tables


def _oracle_window(oracle, packed, pos, tables, pairs, s0, s1, mean_only, post):
    pairs = np.asarray(pairs, np.int32).reshape(-1, 2)
    return oracle.fb_window(packed, pos, s0, s1 - s0, pairs[:, 0], pairs[:, 1], NE, tables,
                            ci=not mean_only, posterior=post)


def test_run_fb_window_matches_oracle(small_ctx, oracle):
    ctx, G, pos, packed, tables = small_ctx
    S = G.shape[1]
    pairs = synthetic.all_pairs(G.shape[0])[::7]
    for s0, s1 in ((0, S), (0, 1), (1, 2), (0, 300), (1000, S), (S - 1, S), (517, 1733)):
        got = ctx.run_fb_window(pairs, s0, s1, mean_only=False, return_posterior=True)
        want = _oracle_window(oracle, packed, pos, tables, pairs, s0, s1, False, True)
        _check(got, want)
    full = ctx.run_fb(pairs, mean_only=False, return_posterior=True)
    _check(ctx.run_fb_window(pairs, 0, S, mean_only=False, return_posterior=True), full)
    empty = ctx.run_fb_window(pairs, 5, 5)
    assert empty["mean"].shape == (0, len(pairs))
    with pytest.raises(ValueError, match="out of range"):
        ctx.run_fb_window(pairs, 10, S + 1)


def _mixed_jobs(rng, n_haps, S, n_jobs):
    allp = synthetic.all_pairs(n_haps)
    jobs = []
    for k in range(n_jobs):
        n = int(rng.integers(1, min(300, len(allp)) + 1))
        pairs = allp[rng.choice(len(allp), n, replace=False)]
        w = int(rng.integers(1, S + 1))
        s0 = int(rng.integers(0, S - w + 1))
        mode = k % 3
        jobs.append(Job(pairs, s0, s0 + w, mean_only=mode != 1, return_posterior=mode == 2))
    return jobs


@pytest.mark.parametrize("width,ppt,graph", [(32, 1, True), (32, 2, False), (128, 1, True),
                                              (128, 2, True), (32, 1, False)])
def test_jobs_match_oracle_every_shape(small_ctx, oracle, width, ppt, graph):
    ctx, G, pos, packed, tables = small_ctx
    rng = np.random.default_rng(11 + width + ppt)
    jobs = _mixed_jobs(rng, G.shape[0], G.shape[1], 40)
    jobs.append(Job(np.zeros((0, 2), np.int32), 0, 10))       # no pairs
    jobs.append(Job([(3, 1)], 7, 7))                           # empty window
    got = run_jobs(ctx, jobs, tile_width=width, pairs_per_thread=ppt, use_graph=graph)
    assert len(got) == len(jobs)
    for j, r in zip(jobs, got):
        want = _oracle_window(oracle, packed, pos, tables, j.pairs, j.site_begin, j.site_end,
                              j.mean_only, j.return_posterior)
        _check(r, want)


def test_executor_reuse_and_two_streams(small_ctx, oracle):
    """Two executors in flight on two streams, each run twice: every result
    equals the oracle's."""
    import torch
    from gamma_smc_cu_b200.batch import DeviceBatch, Layout
    ctx, G, pos, packed, tables = small_ctx
    dev = torch.device("cuda", ctx.device_id)
    rng = np.random.default_rng(5)
    ex = [Executor(ctx, max_window_sites=G.shape[1], max_tasks=4096) for _ in range(2)]
    streams = [torch.cuda.Stream(dev) for _ in range(2)]
    batches = []
    for rnd in range(2):
        for e, st in zip(ex, streams):
            jobs = _mixed_jobs(rng, G.shape[0], G.shape[1], 12)
            b = DeviceBatch(Layout(jobs), dev)
            b.launch(e, st)
            batches.append(b)
    for b in batches:
        for j, r in zip(b.layout.jobs, b.to_host()):
            want = _oracle_window(oracle, packed, pos, tables, j.pairs, j.site_begin,
                                  j.site_end, j.mean_only, j.return_posterior)
            _check(r, want)
    for e in ex:
        e.close()


@pytest.mark.parametrize("flank", [2048, 4])
def test_chunked_jobs_equal_whole_windows(oracle, flow_field, flank):
    """Long windows cut into 2,048-site chunks equal the unchunked decode bit
    for bit: the chunks' boundary states are checked on the device and a job
    that fails the check (forced here by a 4-site burn-in) is decoded again
    whole."""
    import torch
    from gamma_smc_cu_b200.batch import DeviceBatch, Layout, _count_tasks
    G, pos = synthetic.cohort("chrom", n_sites=12000)
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, NE)
    ctx = _core.FlowContext(G, pos, NE, mu, rho, flow_field, 0)
    rng = np.random.default_rng(2)
    allp = synthetic.all_pairs(G.shape[0])
    jobs = []
    for k in range(12):
        n = int(rng.integers(1, 200))
        w = int(rng.integers(3000, 12001))
        s0 = int(rng.integers(0, 12000 - w + 1))
        jobs.append(Job(allp[rng.choice(len(allp), n, replace=False)], s0, s0 + w,
                        mean_only=k % 2 == 0, return_posterior=k % 4 == 1))
    cfg = dict(core_block_sites=2048, flank_sites=flank)
    ex = Executor(ctx, max_tasks=_count_tasks(jobs, cfg) + 8, **cfg)
    b = DeviceBatch(Layout(jobs), ctx.device_id)
    b.launch(ex, torch.cuda.current_stream(torch.device("cuda", ctx.device_id)))
    chunked = b.to_host()
    if flank == 4:
        assert b.repaired > 0
    for j, r in zip(jobs, chunked):
        want = ctx.run_fb_window(j.pairs, j.site_begin, j.site_end, mean_only=j.mean_only,
                                 return_posterior=j.return_posterior)
        _check(r, want, exact=True)
    ex.close()
    if flank == 2048:
        for j, r in zip(jobs, run_jobs(ctx, jobs, **cfg)):
            _check(r, ctx.run_fb_window(j.pairs, j.site_begin, j.site_end, mean_only=j.mean_only,
                                        return_posterior=j.return_posterior), exact=True)


def test_job_errors(small_ctx):
    ctx, G, pos, packed, tables = small_ctx
    S = G.shape[1]
    with pytest.raises(ValueError, match="out of range"):
        run_jobs(ctx, [Job([(1, 0)], 0, S + 1)])
    with pytest.raises(ValueError, match="pair index out of range"):
        run_jobs(ctx, [Job([(40, 0)], 0, 10)])
    ex = Executor(ctx, max_window_sites=100, max_tasks=4)
    with pytest.raises(ValueError, match="max_window_sites"):
        run_jobs(ctx, [Job([(1, 0)], 0, 101)], executor=ex)
    with pytest.raises(ValueError, match="max_tasks"):
        run_jobs(ctx, [Job([(1, 0)], 0, 10)] * 5, executor=ex)
    ex.close()
