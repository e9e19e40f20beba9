"""Small, self-contained runs of each kernel, for profilers.

    python -m gamma_smc_cu_b200.profile_cases <case> [--repeat N]

Each case builds its inputs, runs the kernel once to warm up and then
``--repeat`` more times, and exits; sizes keep the inputs/outputs above the
126 MB L2 of a B200 (so DRAM counters mean something) while holding at most a
few GB on the device.  Cases:

* ``scan``      cached FB, chromosome cohort, 8,192 sites x 63,190 pairs,
                blockwise core 512 / flank 128 (16 windows x 247 tiles of 256
                pairs: enough tasks for the two-pairs-per-thread shape the
                full chromosome job runs), mean-only
* ``full``      cached FB with the full posterior (mean + alpha + beta, the
                output-write-bound mode), chromosome cohort, 4,096 sites x
                63,190 pairs, blockwise core 256 / flank 64 (16 windows: the
                two-pairs-per-thread shape)
* ``batch``     64 uneven jobs (1-2,000 pairs, 2k-40k-site windows) over a
                60,000-site slice of the chromosome cohort, one executor launch
                (32-thread tiles, 4,096-site chunks)
* ``summary``   per-site summary over 16,384 pairs x 20,000 sites (blockwise
                8,192 / 2,048)
* ``fwd``       forward-only posterior, 8,192 pairs x 20,000 sites
* ``uncached``  uncached flow-field FB, 4,096 pairs x 10,000 sites
* ``flowgen``   GPU flow-field generation, 51 x 50 cells, constant Ne
* ``fwd_spec``  forward-only posterior, 2,000 pairs x 400,000 sites (few pairs:
                the sites run in exact speculative chunks)
* ``uncached_spec`` uncached flow-field FB, 500 pairs x 200,000 sites (same)
"""
from __future__ import annotations

import argparse

import numpy as np


def _ctx(n_sites):
    from . import _core, synthetic
    from .infer import _estimate_scaled_params
    G, pos = synthetic.cohort("chrom", n_sites=n_sites)
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    return _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0), G, pos


def case_scan(repeat):
    import torch
    from . import _lib, synthetic
    ctx, G, pos = _ctx(8192)
    pairs = synthetic.all_pairs(G.shape[0])
    dev = torch.device("cuda", ctx.device_id)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    out = torch.empty((G.shape[1], len(pairs)), device=dev)
    L = _lib.load()
    for _ in range(1 + repeat):
        _lib.check(L.gsmc_run_fb_blockwise_device(
            ctx.handle, pi.data_ptr(), pj.data_ptr(), len(pairs), 512, 128, 0,
            out.data_ptr(), None, None, None, None, len(pairs), 0, None))
    torch.cuda.synchronize()
    print("scan shape", ctx.scan_shape())


def case_full(repeat):
    import torch
    from . import _lib, synthetic
    ctx, G, pos = _ctx(4096)
    pairs = synthetic.all_pairs(G.shape[0])
    dev = torch.device("cuda", ctx.device_id)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    outs = [torch.empty((G.shape[1], len(pairs)), device=dev) for _ in range(3)]
    L = _lib.load()
    for _ in range(1 + repeat):
        _lib.check(L.gsmc_run_fb_blockwise_device(
            ctx.handle, pi.data_ptr(), pj.data_ptr(), len(pairs), 256, 64, _lib.GSMC_POSTERIOR,
            outs[0].data_ptr(), None, None, outs[1].data_ptr(), outs[2].data_ptr(), len(pairs), 0,
            None))
    torch.cuda.synchronize()
    print("scan shape", ctx.scan_shape())


def case_batch(repeat):
    import torch
    from .batch import DeviceBatch, Executor, Job, Layout, _count_tasks
    from . import synthetic
    ctx, G, pos = _ctx(60000)
    jobs = [Job(**j) for j in synthetic.job_mix(G.shape[0], G.shape[1], 64, seed=5,
                                                 pairs_range=(1, 2000),
                                                 window_range=(2000, 40000))]
    cfg = dict(tile_width=32, pairs_per_thread=1, core_block_sites=4096, flank_sites=2048)
    ex = Executor(ctx, max_tasks=_count_tasks(jobs, cfg) + 16, **cfg)
    st = torch.cuda.Stream(torch.device("cuda", ctx.device_id))
    b = DeviceBatch(Layout(jobs), ctx.device_id)
    b.allocate(st)
    with torch.cuda.stream(st):
        b.d_pairs.copy_(b.h_pairs, non_blocking=True)
    for _ in range(1 + repeat):
        ex.run(b.layout, b.d_pairs.data_ptr(), b.d_out.data_ptr(), st.cuda_stream)
    st.synchronize()
    ex.close()


def case_summary(repeat):
    from . import synthetic
    ctx, G, pos = _ctx(20000)
    pairs = synthetic.random_pairs(G.shape[0], 16384, 3)
    for _ in range(1 + repeat):
        ctx.run_fb_summary(pairs, core_block_sites=8192, flank_sites=2048)


def case_fwd(repeat):
    from . import synthetic
    ctx, G, pos = _ctx(20000)
    pairs = synthetic.random_pairs(G.shape[0], 8192, 4)
    for _ in range(1 + repeat):
        ctx.run_fwd(pairs)


def case_uncached(repeat):
    from . import _core, synthetic
    G, pos = synthetic.cohort("chrom", n_sites=10000)
    pairs = synthetic.random_pairs(G.shape[0], 4096, 6)
    for _ in range(1 + repeat):
        _core.gamma_smc_flow_fb(G, pos, pairs, mean_only=True)


def case_flowgen(repeat):
    from .demographic import generate_flow_field
    for _ in range(1 + repeat):
        generate_flow_field(verbose=False)


def case_fwd_spec(repeat):
    from . import synthetic
    ctx, G, pos = _ctx(400000)
    pairs = synthetic.random_pairs(G.shape[0], 2000, 4)
    for _ in range(1 + repeat):
        ctx.run_fwd(pairs)


def case_uncached_spec(repeat):
    from . import _core, synthetic
    G, pos = synthetic.cohort("chrom", n_sites=200000)
    pairs = synthetic.random_pairs(G.shape[0], 500, 4)
    for _ in range(1 + repeat):
        _core.gamma_smc_flow_fb(G, pos, pairs, mean_only=True)


CASES = {"scan": case_scan, "full": case_full, "batch": case_batch, "summary": case_summary, "fwd": case_fwd,
         "uncached": case_uncached, "flowgen": case_flowgen, "fwd_spec": case_fwd_spec,
         "uncached_spec": case_uncached_spec}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    CASES[a.case](a.repeat)
    print(f"{a.case}: ok")


if __name__ == "__main__":
    main()
