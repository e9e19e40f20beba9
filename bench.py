#!/usr/bin/env python
"""Benchmark of the blockwise Gamma-SMC forward/backward scan on 1..N B200s.

Metric: pair-site posteriors per second (pairs x sites / time), whole job.

Workload (default ``chrom``): the chromosome-shape cohort -- 356 haplotypes
(63,190 pairs) x 400,000 segregating sites, synthetic (seeded copying-mosaic
genotypes; msprime is unavailable) -- decoded blockwise with
core_block_sites = the API's auto choice on a B200 (32,768), flank_sites=2048,
mean_only=True.  One step = one pass over the whole job.

* ``value``: device-resident -- genotypes, tables and pair indices already in
  HBM, the [n_sites x n_pairs] float32 output written to HBM (101 GB, far
  larger than L2, so no flush is needed), timed with CUDA events.
* ``e2e``: the same job through the public API with host buffers
  (``FlowContext(G, positions, ...)`` + ``run_fb_blockwise`` into numpy), so
  the H2D of the genotypes and the D2H of every posterior are inside the
  timed region.
* ``roofline``: the scan kernel's algorithmic bytes (4 B mean + 0.25 B of
  genotype bits per pair-site) over its event-timed duration, against the
  measured HBM copy bandwidth.
* ``cpu_baseline``: the CPU oracle (a C++ restatement of the reference's scan,
  OpenMP over pairs) on a bounded sample of the same workload.

``--impl reference`` times the reference path's CPU implementation (the
oracle port: the reference ships no CPU scan) on the host cores instead.
Multi-GPU: one process per GPU (torchrun); each rank decodes its own cohort
(weak scaling), no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "pair-site posteriors/sec"
UNIT = "pair-sites/s"
BYTES_MEAN_ONLY = 4.25      # 4 B fp32 mean + 2 genotype bits per pair-site
BYTES_FULL_POSTERIOR = 12.25
# DRAM bytes (read + write) the scan kernel moves per core pair-site in
# mean-only mode, from an ncu capture of the same kernel on the first 8,192
# sites x 63,190 pairs (`--case scan`): 16 B forward-state round trip + 4 B
# output.
TRAFFIC_PER_PAIR_SITE = 20.0
# The same for the full posterior (mean + alpha + beta), from an ncu capture
# of the 50,000-site slice's launch shape on 8,192 pairs (`--case
# full_slice`): 11.44 GB over 4.1e8 core pair-sites -- 12 B of outputs, the
# 16 B forward-state round trip, and the speculative chunks' burn-in reads.
TRAFFIC_FULL_PER_PAIR_SITE = 28.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="chrom", choices=["chrom", "small", "chromprof"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-full-posterior", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-summary", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU build on the same jobs")
    ap.add_argument("--no-stress", action="store_true",
                    help="skip the 2,000-haplotype x 1,000,000-pair streamed run")
    ap.add_argument("--plain-jobs", type=int, default=48,
                    help="jobs of the mix timed through the plain per-call path")
    ap.add_argument("--case", default=None,
                    help="run one small profiling case instead of the benchmark")
    ap.add_argument("--repeat", type=int, default=1, help="repetitions of --case")
    ap.add_argument("--reference-gpu-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--watchdog", type=float, default=900.0,
                    help="dump every thread's stack to stderr every this many seconds (0: off)")
    return ap.parse_args()


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def l2_note(out_bytes):
    """How the timed steps stand to the 126 MB L2: the mean-only output alone."""
    if out_bytes > 126e6:
        return f"output {out_bytes / 1e9:.2f} GB > L2 (no flush needed)"
    return f"output {out_bytes / 1e6:.1f} MB fits L2 (parity-size case, not flushed)"


def workload(name, rank):
    from gamma_smc_cu_b200 import synthetic
    if name == "small":
        G, pos = synthetic.cohort("small")
        pairs = synthetic.all_pairs(G.shape[0])
        return G, pos, pairs, G.shape[1], 0, "small: 40 haps x 2,127 sites x 780 pairs"
    if name == "chromprof":
        # profiling case with the chrom launch shape (all 63,190 pairs, several
        # windows per launch) on 6,144 sites: core 2048, flank 1024 -> 3 windows,
        # 1.55 GB output (> L2) + 3.1 GB forward states
        G, pos = synthetic.cohort("chrom", n_sites=6144)
        pairs = synthetic.all_pairs(G.shape[0])
        return G, pos, pairs, 2048, 1024, "chromprof: 356 haps x 6,144 sites x 63,190 pairs"
    n, S, _, sp, sg = synthetic.COHORTS["chrom"]
    span = synthetic.neutral_span(n, S)
    pos = synthetic.positions_for(S, span, sp + 100 * rank)
    G = synthetic.haplotypes(n, pos, sg + 100 * rank)
    pairs = synthetic.all_pairs(n)
    return G, pos, pairs, None, 2048, "chrom: 356 haps x 400,000 sites x 63,190 pairs"


def cpu_baseline_sample(G, pos, pairs, core, flank, mu, rho, target_s=12.0):
    """Time the CPU oracle on a bounded pair sample of the same job."""
    from oracle import oracle as O
    from gamma_smc_cu_b200._core import DEFAULT_FLOW_FIELD
    threads = os.cpu_count() or 1
    O.tables_for(DEFAULT_FLOW_FIELD, 1e4, mu, rho)
    S = G.shape[1]
    # grow the pair sample until one run takes a few seconds, at most ~target_s
    n = min(len(pairs), max(4 * threads, 64))
    while True:
        t0 = time.perf_counter()
        O.run_fb_blockwise(G, pos, [tuple(p) for p in pairs[:n]], 1e4, mu, rho,
                           DEFAULT_FLOW_FIELD, core, flank, True, False, threads)
        dt = time.perf_counter() - t0
        if dt >= target_s / 3 or n >= len(pairs):
            break
        n = min(len(pairs), int(n * min(8.0, max(2.0, target_s / max(dt, 1e-3)))))
    return {"value": n * S / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} pairs x {S} sites, blockwise core={core} flank={flank}, "
                      f"mean_only, {dt:.1f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    G, pos, pairs, core, flank, desc = workload(args.workload, 0)
    from gamma_smc_cu_b200.infer import _estimate_scaled_params, _recommend_core_block_size
    from oracle import oracle as O
    from gamma_smc_cu_b200._core import DEFAULT_FLOW_FIELD
    S = G.shape[1]
    if core is None:
        core, _ = _recommend_core_block_size(S, len(pairs), True, flank, 178 * 10**9)
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    threads = os.cpu_count() or 1
    O.tables_for(DEFAULT_FLOW_FIELD, 1e4, mu, rho)
    # A step is a bounded pair sample of the job: at least 4,096 pairs (enough
    # work per thread that every host core stays busy to the end) and at least
    # ~8 s of CPU work, sized from a 256-pair probe.
    probe = pairs[:min(len(pairs), 256)]
    t0 = time.perf_counter()
    O.run_fb_blockwise(G, pos, [tuple(p) for p in probe], 1e4, mu, rho, DEFAULT_FLOW_FIELD,
                       core, flank, True, False, threads)
    dt = time.perf_counter() - t0
    n_sample = int(min(len(pairs), max(4096, len(probe) * 8.0 / max(dt, 1e-3))))
    sample = [tuple(p) for p in pairs[:n_sample]]
    for _ in range(args.warmup):
        O.run_fb_blockwise(G, pos, sample, 1e4, mu, rho, DEFAULT_FLOW_FIELD, core, flank, True,
                           False, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.run_fb_blockwise(G, pos, sample, 1e4, mu, rho, DEFAULT_FLOW_FIELD, core, flank, True,
                           False, threads)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    value = n_sample * S / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": desc, "core_block_sites": core, "flank_sites": flank,
                       "mean_only": True},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n_sample} pairs x {S} sites per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_T0 = time.perf_counter()


def log(msg):
    """Progress of the run on stderr (the JSON line stays alone on stdout)."""
    sys.stderr.write(f"[bench {time.perf_counter() - _T0:8.1f} s] {msg}\n")
    sys.stderr.flush()


def main():
    args = parse()
    if args.watchdog > 0:
        # if a leg stalls, the stacks of every thread show where
        import faulthandler
        faulthandler.dump_traceback_later(args.watchdog, repeat=True, file=sys.stderr)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.reference_gpu_child:
        reference_gpu_child(args.reference_gpu_child)
        return
    if args.case:
        CASES[args.case](args.repeat)
        print(f"{args.case}: ok")
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import gamma_smc_cu_b200 as G200
    from gamma_smc_cu_b200 import _core, _lib
    from gamma_smc_cu_b200.infer import _estimate_scaled_params, _recommend_core_block_size

    G, pos, pairs, core, flank, desc = workload(args.workload, rank)
    S, P = G.shape[1], len(pairs)
    free, _ = _core.cuda_mem_info()
    if core is None:
        core, _ = _recommend_core_block_size(S, P, True, flank, free)
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    ctx = _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
    L = _lib.load()
    dev = torch.device("cuda", local)
    d_pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    d_pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    out = torch.empty((S, P), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        _lib.check(L.gsmc_run_fb_blockwise_device(
            ctx.handle, d_pi.data_ptr(), d_pj.data_ptr(), P, core, flank, 0, out.data_ptr(),
            None, None, None, None, P, 0, stream.cuda_stream))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _lib.check(L.gsmc_ctx_timing_read(ctx.handle, None, None, None))
    _lib.check(L.gsmc_ctx_timing(ctx.handle, 1))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_ms = e0.elapsed_time(e1)
    import ctypes
    kms = ctypes.c_double()
    launches = ctypes.c_int64()
    psites = ctypes.c_double()
    _lib.check(L.gsmc_ctx_timing_read(ctx.handle, ctypes.byref(kms), ctypes.byref(launches),
                                      ctypes.byref(psites)))
    _lib.check(L.gsmc_ctx_timing(ctx.handle, 0))
    width, ppt = ctypes.c_int(), ctypes.c_int()
    _lib.check(L.gsmc_ctx_scan_shape(ctx.handle, ctypes.byref(width), ctypes.byref(ppt)))
    kernel_name = f"fb_scan_persistent<{ppt.value}, {width.value}, false>"
    if world > 1:
        t = torch.tensor([t_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    ms_per_step = t_ms / args.steps
    value = P * S * world / (t_ms / 1e3 / args.steps)
    hbm, peak_kind = peaks()
    achieved = psites.value * BYTES_MEAN_ONLY / (kms.value / 1e3) / 1e9
    # parity sample: 64 seeded-random pair columns of the timed output, all
    # 400,000 sites, checked against the oracle after the GPU work
    cols = np.sort(np.random.default_rng(11).choice(P, size=min(64, P), replace=False))
    ours_cols = out[:, torch.from_numpy(cols).to(dev)].cpu().numpy()
    del out
    ctx.release_scratch()
    torch.cuda.empty_cache()
    batched = None
    if args.workload == "chrom" and not args.no_batched:
        log("batched")
        batched = run_batched(ctx, G, dev, args.plain_jobs)
    summary = None
    if args.workload == "chrom" and not args.no_summary:
        log("summary")
        summary = run_summary(ctx, pairs, S)
    ctx.close()
    torch.cuda.empty_cache()
    if args.workload == "chrom" and not args.no_batched:
        log("batched small cohort")
        batched["small_cohort"] = run_batched_small(dev)
    traffic = (TRAFFIC_PER_PAIR_SITE * psites.value / launches.value
               if launches.value and args.workload != "small" else None)

    full = None
    if args.workload == "chrom" and not args.no_full_posterior:
        log("full posterior slice")
        full = run_full_posterior(G, pos, pairs, args.steps, args.warmup, dev)

    tables64 = None
    if args.workload == "chrom" and not args.no_full_posterior:
        log("float64 tables")
        tables64 = run_tables_f64(G, pos)

    served = None
    if args.workload == "chrom" and not args.no_served:
        log("served")
        served = run_served(dev)
    stress = None
    if args.workload == "chrom" and not args.no_stress and rank == 0:
        log("stream stress")
        stress = run_stream_stress()

    e2e = None
    if not args.no_e2e:
        log("e2e")
        e2e = run_e2e(G, pos, pairs, core, flank, args.e2e_steps)
    ref_gpu = None
    if args.workload == "chrom" and rank == 0 and not args.no_reference_gpu:
        log("reference GPU build")
        ref_gpu = run_reference_gpu(G, pos, pairs, core, flank, mu, rho, full)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        log("cpu baseline")
        cpu = cpu_baseline_sample(G, pos, pairs, core, flank, mu, rho)
    parity = None
    if rank == 0:
        log("parity")
        parity = {"chrom": oracle_parity(G, pos, pairs[cols], mu, rho, core, flank,
                                         {"mean": ours_cols})}
        if full is not None:
            parity["full_posterior"] = full.pop("parity")
        if stress is not None:
            parity["stream_stress"] = stress.pop("parity")
        parity["exact"] = all(v["exact"] for v in parity.values())
        parity["max_rel"] = max(v["max_rel"] for k, v in parity.items() if isinstance(v, dict))
        parity["pairs_checked"] = sum(v["pairs_checked"] for v in parity.values()
                                      if isinstance(v, dict))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "core_block_sites": int(core), "flank_sites": flank,
                       "mean_only": True, "l2": l2_note(G.shape[1] * len(pairs) * 4),
                       "parallelism": f"pairs replicated per rank x{world} (weak)"},
            "gpu_launches": int(launches.value),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "peak_kind": peak_kind, "kernel": kernel_name,
                         "kernel_ms_per_step": kms.value / args.steps,
                         "bytes_per_pair_site": BYTES_MEAN_ONLY},
            "full_posterior": full,
            "summary": summary,
            "tables_gpu_fp64": tables64,
            "batched": batched,
            "served": served,
            "stream_stress": stress,
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
            "reference_gpu": ref_gpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def timed_device_run(ctx, d_pi, d_pj, P, S, core, flank, flags, outs, steps, warmup, dev):
    """Event-timed device-resident blockwise runs; returns (ms per step,
    kernel ms per step, launches, pair-sites)."""
    import ctypes
    import torch
    from gamma_smc_cu_b200 import _lib
    L = _lib.load()
    stream = torch.cuda.current_stream(dev)
    ptrs = [o.data_ptr() if o is not None else None for o in outs]

    def step():
        _lib.check(L.gsmc_run_fb_blockwise_device(
            ctx.handle, d_pi.data_ptr(), d_pj.data_ptr(), P, core, flank, flags, *ptrs, P, 0,
            stream.cuda_stream))

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    _lib.check(L.gsmc_ctx_timing_read(ctx.handle, None, None, None))
    _lib.check(L.gsmc_ctx_timing(ctx.handle, 1))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    kms = ctypes.c_double()
    launches = ctypes.c_int64()
    psites = ctypes.c_double()
    _lib.check(L.gsmc_ctx_timing_read(ctx.handle, ctypes.byref(kms), ctypes.byref(launches),
                                      ctypes.byref(psites)))
    _lib.check(L.gsmc_ctx_timing(ctx.handle, 0))
    return e0.elapsed_time(e1) / steps, kms.value / steps, launches.value, psites.value


def run_full_posterior(G, pos, pairs, steps, warmup, dev, n_sites=50_000):
    """Full-posterior roofline case: mean + posterior alpha/beta (12.25 B per
    pair-site) on the first 50,000 sites of the chromosome cohort, all pairs,
    blockwise with the API's auto core and flank 2048, outputs in HBM."""
    import torch
    from gamma_smc_cu_b200 import _core, _lib
    from gamma_smc_cu_b200.infer import _estimate_scaled_params, _recommend_core_block_size
    Gs = np.ascontiguousarray(G[:, :n_sites])
    ps = np.ascontiguousarray(pos[:n_sites])
    S, P = Gs.shape[1], len(pairs)
    mu, rho = _estimate_scaled_params(Gs, ps, 1.25e-8, 1e-8, 1e4)
    ctx = _core.FlowContext(Gs, ps, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
    free, _ = _core.cuda_mem_info()
    core, _ = _recommend_core_block_size(S, P, True, 2048, free)
    d_pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    d_pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    outs = [torch.empty((S, P), dtype=torch.float32, device=dev) for _ in range(3)]
    ms, kms, launches, psites = timed_device_run(
        ctx, d_pi, d_pj, P, S, core, 2048, _lib.GSMC_POSTERIOR,
        [outs[0], None, None, outs[1], outs[2]], steps, warmup, dev)
    hbm, kind = peaks()
    steps_ = max(1, steps)
    achieved = psites / steps_ * BYTES_FULL_POSTERIOR / (kms / 1e3) / 1e9
    recon = (outs[1][::997, ::61] / outs[2][::997, ::61]) * 2e4
    ok = bool(torch.allclose(recon, outs[0][::997, ::61], rtol=1e-4, atol=1e-2))
    cols = np.sort(np.random.default_rng(12).choice(P, size=min(64, P), replace=False))
    ct = torch.from_numpy(cols).to(dev)
    got = {k: o[:, ct].cpu().numpy() for k, o in zip(("mean", "posterior_alpha",
                                                       "posterior_beta"), outs)}
    del outs
    shape = ctx.scan_shape()
    spec = ctx.spec_stats()
    ctx.close()
    torch.cuda.empty_cache()
    parity = oracle_parity(Gs, ps, pairs[cols], mu, rho, core, 2048, got, posterior=True)
    return {"workload": f"chrom 50k-site slice: 356 haps x {S} sites x {P} pairs, mean+alpha+beta",
            "core_block_sites": int(core), "flank_sites": 2048, "scan_shape": shape,
            "speculative": spec, "parity": parity, "mu": mu, "rho": rho,
            "value": P * S / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "gpu_launches": int(launches), "posterior_consistent": ok,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": kind,
                         "bytes_per_pair_site": BYTES_FULL_POSTERIOR,
                         "traffic": TRAFFIC_FULL_PER_PAIR_SITE * P * S,
                         "kernel_ms_per_step": kms}}


def oracle_parity(G, pos, pairs, mu, rho, core, flank, got, posterior=False):
    """Bitwise comparison of sampled pair columns (``got``: output name ->
    [n_sites, len(pairs)] float32 from the GPU run) with the CPU oracle run
    blockwise on the same pairs, core and flank.  The oracle is only the
    checker here and runs outside every timed region."""
    from oracle import oracle as O
    from gamma_smc_cu_b200._core import DEFAULT_FLOW_FIELD
    t0 = time.perf_counter()
    want = O.run_fb_blockwise(G, pos, [(int(i), int(j)) for i, j in pairs], 1e4, mu, rho,
                              DEFAULT_FLOW_FIELD, int(core), int(flank), True, posterior,
                              os.cpu_count() or 1)
    exact, mr = True, 0.0
    for k, g in got.items():
        w = want[k][:g.shape[0]]
        exact &= bool(np.array_equal(np.ascontiguousarray(g).view(np.uint32),
                                     np.ascontiguousarray(w).view(np.uint32)))
        mr = max(mr, _max_rel(g, w))
    return {"pairs_checked": int(len(pairs)), "sites": int(next(iter(got.values())).shape[0]),
            "core_block_sites": int(core), "flank_sites": int(flank), "outputs": sorted(got),
            "exact": exact, "max_rel": mr, "oracle_seconds": time.perf_counter() - t0}


def _reference_core():
    """The reference's own _core module, compiled from its sources for sm_100a
    into oracle/_ref by the oracle recipe, or None when it was not built."""
    import importlib.util
    from oracle import oracle as O
    path = O.ref_core_path()
    if path is None:
        return None
    spec = importlib.util.spec_from_file_location("_core", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _cuda_kernel_ms(fn):
    """Run fn() once with CUDA kernel activity recorded (CUPTI, through
    torch.profiler; no replay): (fn's result, {kernel name: total ms})."""
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        r = fn()
    ms = {}
    for e in prof.key_averages():
        t = getattr(e, "device_time_total", None)
        if t is None:
            t = getattr(e, "cuda_time_total", 0.0)
        if t:
            ms[e.key] = ms.get(e.key, 0.0) + t / 1e3
    return r, ms


def _scan_kernel_ms(ms):
    """Total ms of the reference's cached forward/backward kernels."""
    return sum(v for k, v in ms.items() if "gamma_smc_cached" in k or "precompute_xor" in k)


def reference_gpu_child(workdir):
    """Child process of run_reference_gpu: runs the reference's own GPU build
    on the saved inputs, writing each result to results.json as soon as it
    exists (the parent may stop this process at its time limit)."""
    import faulthandler
    from gamma_smc_cu_b200._core import DEFAULT_FLOW_FIELD
    faulthandler.dump_traceback_later(60, repeat=True, file=sys.stderr)
    log("child: loading the reference build")
    ref = _reference_core()
    d = np.load(os.path.join(workdir, "inputs.npz"))
    with open(os.path.join(workdir, "params.json")) as f:
        prm = json.load(f)
    res = {}

    def save():
        with open(os.path.join(workdir, "results.json"), "w") as f:
            json.dump(res, f)

    G, pos = d["G"], d["pos"]
    chrom = [tuple(p) for p in d["chrom_pairs"].tolist()]
    core, flank = prm["core"], prm["flank"]
    log(f"child: FlowContext {G.shape}")
    t0 = time.perf_counter()
    ctx = ref.FlowContext(G, pos, 1e4, prm["mu"], prm["rho"], DEFAULT_FLOW_FIELD, 0)
    res["chrom_context_seconds"] = time.perf_counter() - t0
    log(f"child: run_fb_blockwise {len(chrom)} pairs")
    r = ref.FlowContext.run_fb_blockwise(ctx, chrom, core, flank, -1, 1, True, False)
    res["chrom_seconds"] = time.perf_counter() - t0
    log(f"child: done {res['chrom_seconds']:.1f} s")
    np.save(os.path.join(workdir, "chrom_cols.npy"), np.ascontiguousarray(r["mean"][:, :64]))
    del r
    save()
    del ctx
    n = prm["slice_sites"]
    Gs, ps = np.ascontiguousarray(G[:, :n]), np.ascontiguousarray(pos[:n])
    sl = [tuple(p) for p in d["slice_pairs"].tolist()]
    t0 = time.perf_counter()
    ctx = ref.FlowContext(Gs, ps, 1e4, prm["slice_mu"], prm["slice_rho"], DEFAULT_FLOW_FIELD, 0)
    r = ref.FlowContext.run_fb(ctx, sl, True, True)
    res["slice_seconds"] = time.perf_counter() - t0
    log(f"child: slice {res['slice_seconds']:.1f} s")
    np.savez(os.path.join(workdir, "slice_cols.npz"),
             **{k: np.ascontiguousarray(r[k][:, :64])
                for k in ("mean", "posterior_alpha", "posterior_beta")})
    del r
    save()
    r, ms = _cuda_kernel_ms(lambda: ref.FlowContext.run_fb(ctx, sl, True, True))
    del r, ctx
    res["slice_kernel_ms"] = _scan_kernel_ms(ms)
    save()
    log("child: chromosome kernels")
    ctx = ref.FlowContext(G, pos, 1e4, prm["mu"], prm["rho"], DEFAULT_FLOW_FIELD, 0)
    r, ms = _cuda_kernel_ms(lambda: ref.FlowContext.run_fb_blockwise(
        ctx, chrom, core, flank, -1, 1, True, False))
    del r, ctx
    res["chrom_kernel_ms"] = _scan_kernel_ms(ms)
    res["chrom_by_kernel_ms"] = {k: v for k, v in sorted(ms.items(), key=lambda kv: -kv[1])[:6]}
    save()


def run_reference_gpu(G, pos, pairs, core, flank, mu, rho, full, chrom_pairs=128,
                      slice_pairs=512, slice_sites=50_000, time_limit=150.0):
    """Informational: the reference's own GPU build (its pybind11 _core from
    the reference sources, compiled for sm_100a) on the same box, through its
    public FlowContext API with host outputs, on bounded samples: the first
    128 pairs of the chromosome job over all 400,000 sites (blockwise, the
    same core and flank), and 512 pairs of the 50,000-site full-posterior
    slice (run_fb with alpha/beta).  It runs in a child process stopped after
    `time_limit` seconds (the full 63,190-pair job through it did not finish
    within 23 minutes here); its kernel-only times come from CUDA activity
    records of a second run.  This build's same calls run beside it, wall
    clock and kernel events, and the first 64 pairs' columns are compared
    bitwise."""
    import shutil
    import tempfile
    from gamma_smc_cu_b200 import _core, _lib
    from gamma_smc_cu_b200._core import DEFAULT_FLOW_FIELD
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    from oracle import oracle as O
    if O.ref_core_path() is None:
        return {"unavailable": "the reference _core was not built into oracle/_ref"}
    S = G.shape[1]
    cp = np.ascontiguousarray(pairs[:chrom_pairs])
    sp = np.ascontiguousarray(pairs[:slice_pairs])
    Gs, ps = np.ascontiguousarray(G[:, :slice_sites]), np.ascontiguousarray(pos[:slice_sites])
    if full is not None:
        smu, srho = full["mu"], full["rho"]
    else:
        smu, srho = _estimate_scaled_params(Gs, ps, 1.25e-8, 1e-8, 1e4)
    work = tempfile.mkdtemp(prefix="gsmc_refgpu_")
    out = {"build": "reference sources, nvcc 12.9 -gencode arch=compute_100a,code=sm_100a "
                    "(its own CMake targets sm_80)", "time_limit_s": time_limit}
    try:
        np.savez(os.path.join(work, "inputs.npz"), G=G, pos=pos, chrom_pairs=cp, slice_pairs=sp)
        with open(os.path.join(work, "params.json"), "w") as f:
            json.dump({"core": int(core), "flank": int(flank), "mu": mu, "rho": rho,
                       "slice_sites": slice_sites, "slice_mu": smu, "slice_rho": srho}, f)
        status = "finished"
        err = b""
        try:
            p = subprocess.run([sys.executable, os.path.abspath(__file__), "--reference-gpu-child",
                                work], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                               timeout=time_limit)
            err = p.stderr or b""
            if p.returncode != 0:
                status = f"exited {p.returncode}"
        except subprocess.TimeoutExpired as e:
            status = f"stopped at the {time_limit:.0f} s limit"
            err = e.stderr or b""
        out["status"] = status
        lines = [l for l in err.decode(errors="replace").splitlines() if l.strip()]
        out["child_log"] = [l for l in lines if l.startswith("[bench")][-12:]
        sys.stderr.write("\n".join(lines[-60:]) + "\n")
        rpath = os.path.join(work, "results.json")
        res = json.load(open(rpath)) if os.path.exists(rpath) else {}

        def ours(ctx, fn):
            _lib.check(_lib.load().gsmc_ctx_timing_read(ctx.handle, None, None, None))
            _lib.check(_lib.load().gsmc_ctx_timing(ctx.handle, 1))
            r = fn()
            kms = ctypes_double()
            _lib.check(_lib.load().gsmc_ctx_timing_read(ctx.handle, kms.ref(), None, None))
            _lib.check(_lib.load().gsmc_ctx_timing(ctx.handle, 0))
            return r, kms.value

        t0 = time.perf_counter()
        ctx = _core.FlowContext(G, pos, 1e4, mu, rho, DEFAULT_FLOW_FIELD, 0)
        r, kms = ours(ctx, lambda: ctx.run_fb_blockwise(
            [tuple(x) for x in cp.tolist()], core_block_sites=int(core), flank_sites=int(flank),
            pair_batch_size=len(cp), max_streams=1, mean_only=True))
        t_ours = time.perf_counter() - t0
        job = {"workload": f"chrom: first {len(cp)} pairs x {S} sites, blockwise core {core} / "
                           f"flank {flank}, mean_only, host outputs",
               "ours_seconds": t_ours, "ours_kernel_ms": kms}
        cpath = os.path.join(work, "chrom_cols.npy")
        if os.path.exists(cpath):
            job["sampled_columns_bit_equal"] = bool(np.array_equal(
                np.load(cpath).view(np.uint32), np.ascontiguousarray(r["mean"][:, :64]).view(np.uint32)))
        del r
        ctx.close()
        if "chrom_seconds" in res:
            job.update({"seconds": res["chrom_seconds"],
                        "value": len(cp) * S / res["chrom_seconds"], "unit": UNIT,
                        "speedup_wall": res["chrom_seconds"] / t_ours})
        if res.get("chrom_kernel_ms"):
            job.update({"kernel_ms": res["chrom_kernel_ms"],
                        "kernel_pair_sites_per_s": len(cp) * S / (res["chrom_kernel_ms"] / 1e3),
                        "kernel_speedup": res["chrom_kernel_ms"] / kms,
                        "by_kernel_ms": res.get("chrom_by_kernel_ms")})
        out["chrom"] = job
        t0 = time.perf_counter()
        ctx = _core.FlowContext(Gs, ps, 1e4, smu, srho, DEFAULT_FLOW_FIELD, 0)
        r, kms = ours(ctx, lambda: ctx.run_fb([tuple(x) for x in sp.tolist()], mean_only=True,
                                              return_posterior=True))
        t_ours = time.perf_counter() - t0
        sl = {"workload": f"chrom {slice_sites}-site slice: first {len(sp)} pairs, run_fb "
                          "mean + alpha + beta, host outputs",
              "ours_seconds": t_ours, "ours_kernel_ms": kms}
        spath = os.path.join(work, "slice_cols.npz")
        if os.path.exists(spath):
            want = np.load(spath)
            sl["sampled_columns_bit_equal"] = all(
                np.array_equal(want[k].view(np.uint32),
                               np.ascontiguousarray(r[k][:, :64]).view(np.uint32))
                for k in ("mean", "posterior_alpha", "posterior_beta"))
        del r
        ctx.close()
        if "slice_seconds" in res:
            sl.update({"seconds": res["slice_seconds"],
                       "value": len(sp) * slice_sites / res["slice_seconds"], "unit": UNIT,
                       "speedup_wall": res["slice_seconds"] / t_ours})
        if res.get("slice_kernel_ms"):
            sl.update({"kernel_ms": res["slice_kernel_ms"],
                       "kernel_speedup": res["slice_kernel_ms"] / kms})
        out["full_posterior"] = sl
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return out


class ctypes_double:
    """A double out-parameter for the ctypes calls above."""

    def __init__(self):
        import ctypes
        self._v = ctypes.c_double()
        self._ref = ctypes.byref(self._v)

    def ref(self):
        return self._ref

    @property
    def value(self):
        return float(self._v.value)


def _max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


BATCH_WORKLOAD = ("512 jobs (seed 5) over the chromosome cohort: pairs log-uniform "
                  "[1, 4096], windows log-uniform [1e3, 2e5] sites, mean_only")


def run_batched(ctx, G, dev, plain_jobs, jobs=None, workload=BATCH_WORKLOAD):
    """Uneven batch: by default 512 jobs (seed 5) over the chromosome cohort
    -- pair count log-uniform in [1, 4096], window log-uniform in [1e3, 2e5]
    sites -- in one persistent launch with the autotuned launch shape and
    sites-per-chunk, against the plain per-call path (one
    FlowContext.run_fb_window call per job, host outputs) on the first
    ``plain_jobs`` jobs."""
    import torch
    from gamma_smc_cu_b200 import synthetic
    from gamma_smc_cu_b200.batch import DeviceBatch, Executor, Job, Layout, _count_tasks
    from gamma_smc_cu_b200.tune import autotune, executor_kwargs
    if jobs is None:
        jobs = [Job(**j) for j in synthetic.job_mix(G.shape[0], G.shape[1], 512, seed=5)]
    total = float(sum(j.pair_sites for j in jobs))
    t0 = time.perf_counter()
    tuned = autotune(ctx, jobs, use_cache=False)
    tune_s = time.perf_counter() - t0
    kw = executor_kwargs(tuned)
    ex = Executor(ctx, max_tasks=_count_tasks(jobs, kw) + 16, use_graph=True, **kw)
    st = torch.cuda.Stream(dev)
    # device-resident: pairs uploaded, outputs stay in HBM
    b = DeviceBatch(Layout(jobs), dev)
    b.allocate(st)
    with torch.cuda.stream(st):
        b.d_pairs.copy_(b.h_pairs, non_blocking=True)
    run = lambda: ex.run(b.layout, b.d_pairs.data_ptr(), b.d_out.data_ptr(), st.cuda_stream,
                         flags=b.d_flags.data_ptr())   # chunked jobs checked on the device
    for _ in range(2):
        run()
    st.synchronize()
    ex.timing(True)
    ex.timing_read()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 3
    e0.record(st)
    for _ in range(reps):
        run()
    e1.record(st)
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    kms, launches, _ = ex.timing_read()
    ex.timing(False)
    del b
    torch.cuda.empty_cache()
    # end to end on the sample the plain path is timed on: host pairs in,
    # host numpy results out, one launch for all jobs vs one call per job
    sample = jobs[:plain_jobs]
    sample_ps = float(sum(j.pair_sites for j in sample))
    for rep in range(2):   # the first pass warms the allocators
        t0 = time.perf_counter()
        bs = DeviceBatch(Layout(sample), dev)
        bs.launch(ex, st)
        got = bs.to_host()
        batched_s = time.perf_counter() - t0
        del bs
    # the same batch with its results landing by DMA in a pinned buffer that
    # is reused batch after batch (the server's result arena): the results are
    # views into it, so no host thread copies or page-faults them
    from gamma_smc_cu_b200.serve import PinnedArena
    arena = PinnedArena(Layout(sample).out_floats * 4 + (1 << 20))
    for rep in range(3):
        t0 = time.perf_counter()
        bs = DeviceBatch(Layout(sample), dev)
        bs.launch(ex, st, host=arena.alloc(bs.layout.out_floats * 4))
        got_pinned = bs.results()
        pinned_s = time.perf_counter() - t0
        err_pinned = max(_max_rel(g["mean"], w["mean"]) for g, w in zip(got_pinned, got))
        del bs, got_pinned
    big = max(sample, key=lambda j: j.pair_sites)   # grow the per-call scratch first
    ctx.run_fb_window(big.pairs, big.site_begin, big.site_end)
    t0 = time.perf_counter()
    want = [ctx.run_fb_window(j.pairs, j.site_begin, j.site_end) for j in sample]
    plain_s = time.perf_counter() - t0
    # the plain per-call path with page-locked result buffers too (second pass:
    # the first one fills the buffer cache)
    from gamma_smc_cu_b200 import _core, _lib
    prev = _core.set_result_memory("pinned")
    try:
        for rep in range(2):
            t0 = time.perf_counter()
            for j in sample:
                r = ctx.run_fb_window(j.pairs, j.site_begin, j.site_end)
                del r
            plain_pinned_s = time.perf_counter() - t0
    finally:
        _core.set_result_memory(prev)
        _lib.check(_lib.load().gsmc_host_cache_limit(0))        # give the memory back
        _lib.check(_lib.load().gsmc_host_cache_limit(256 << 30))
    err = max(_max_rel(g["mean"], w["mean"]) for g, w in zip(got, want))
    ex.close()
    return {"workload": workload, "pair_sites": total, "device_ms": dev_ms, "kernel_ms": kms / max(1, reps),
            "value": total / (dev_ms / 1e3), "unit": UNIT, "gpu_launches_per_batch": 1,
            "tuned": {k: tuned[k] for k in ("tile_width", "pairs_per_thread",
                                            "core_block_sites", "flank_sites")},
            "tune_seconds": tune_s, "tune_trials": tuned["searched"],
            "sample_jobs": len(sample), "sample_pair_sites": sample_ps,
            "sample_batched_e2e": sample_ps / batched_s,
            "sample_batched_pinned_e2e": sample_ps / pinned_s,
            "sample_plain_per_call": sample_ps / plain_s,
            "sample_plain_per_call_pinned": sample_ps / plain_pinned_s,
            "speedup_vs_plain": plain_s / pinned_s,
            "speedup_vs_plain_numpy_out": plain_s / batched_s,
            "speedup_vs_plain_pinned": plain_pinned_s / pinned_s,
            "max_rel_mean_vs_plain": max(err, err_pinned)}


def run_tables_f64(G, pos, n_sites=50_000, n_pairs=4096):
    """The optional float64 GPU table build against the bit-exact host float32
    build: build seconds of each, and the posterior-mean deviation
    (max relative) of the same calls through the two table sets -- the small
    cohort's 780 pairs over its whole sequence, and 4,096 pairs of the
    chromosome cohort's first 50,000 sites."""
    from gamma_smc_cu_b200 import _core, synthetic
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    out = {}
    Gs, ps = synthetic.cohort("small")
    cases = [("small cohort, 780 pairs x 2,127 sites", Gs, ps, synthetic.all_pairs(Gs.shape[0])),
             (f"chrom {n_sites}-site slice, {n_pairs} pairs",
              np.ascontiguousarray(G[:, :n_sites]), np.ascontiguousarray(pos[:n_sites]),
              synthetic.random_pairs(G.shape[0], n_pairs, 41))]
    for name, Gc, pc, pairs in cases:
        mu, rho = _estimate_scaled_params(Gc, pc, 1.25e-8, 1e-8, 1e4)
        _core.free_cached_tables()
        res = {}
        for build in ("host_fp32", "gpu_fp64"):
            ctx = _core.FlowContext(Gc, pc, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0,
                                    table_build=build)
            secs = ctx.tables_info()["build_seconds"]
            res[build] = (secs, ctx.run_fb(pairs, mean_only=True)["mean"])
            ctx.close()
        a, b = res["host_fp32"][1].astype(np.float64), res["gpu_fp64"][1].astype(np.float64)
        rel = np.abs(b - a) / np.abs(a)
        out[name] = {"build_seconds_host_fp32": res["host_fp32"][0],
                     "build_seconds_gpu_fp64": res["gpu_fp64"][0],
                     "mean_max_rel": float(rel.max()), "mean_median_rel": float(np.median(rel)),
                     "within_1e-4": bool(rel.max() <= 1e-4)}
    _core.free_cached_tables()
    return out


def run_summary(ctx, pairs, S, steps=2):
    """FlowContext.run_fb_summary(pairs) over the whole chromosome job (the
    reference's default: one full-sequence window), host arrays out: per-site
    mean / min / max over all 63,190 pairs, wall clock per call."""
    plist = [tuple(p) for p in pairs.tolist()]
    r = ctx.run_fb_summary(plist)                      # warm-up
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        r = ctx.run_fb_summary(plist)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    ok = bool(np.all(r["site_min"] <= r["site_mean"]) and np.all(r["site_mean"] <= r["site_max"]))
    return {"workload": f"run_fb_summary, full sequence: {S} sites x {len(plist)} pairs",
            "seconds": t, "value": len(plist) * S / t, "unit": UNIT, "consistent": ok}


def run_batched_small(dev):
    """The same 512-job mix (seed 5) over the small cohort (40 haplotypes,
    2,127 sites over 1 Mb): pair counts log-uniform in [1, 4096] clamped to
    its 780 pairs, windows log-uniform in [1 kb, 200 kb] of sequence (1-436
    sites); batched in one launch against all 512 jobs one call each."""
    from gamma_smc_cu_b200 import _core, synthetic
    from gamma_smc_cu_b200.batch import Job
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    G, pos = synthetic.cohort("small")
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    ctx = _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
    jobs = [Job(**j) for j in synthetic.job_mix_bp(pos, G.shape[0], 512, seed=5)]
    try:
        return run_batched(ctx, G, dev, len(jobs), jobs=jobs, workload=(
            "512 jobs (seed 5) over the small cohort (40 haps x 2,127 sites, 1 Mb): pairs "
            "log-uniform [1, 4096] clamped to 780, windows log-uniform [1 kb, 200 kb] "
            "(1-436 sites), mean_only"))
    finally:
        ctx.close()


def _plain_latency(ctx, reqs, pos):
    """Serve ``reqs`` one call at a time in arrival order (FIFO, real time);
    returns (latencies s, pair-sites, wall s)."""
    t0 = time.perf_counter()
    lat = []
    ps = 0.0
    for r in reqs:
        now = time.perf_counter() - t0
        if r["t"] > now:
            time.sleep(r["t"] - now)
        s0 = int(np.searchsorted(pos, r["region_bp"][0]))
        s1 = max(s0, int(np.searchsorted(pos, r["region_bp"][1])))
        ctx.run_fb_window(r["pairs"], s0, s1, mean_only=r["mean_only"],
                          return_posterior=r["return_posterior"])
        lat.append(time.perf_counter() - t0 - r["t"])
        ps += len(r["pairs"]) * (s1 - s0)
    return np.array(lat), ps, time.perf_counter() - t0


def _served_latency(srv, reqs):
    """Submit ``reqs`` at their arrival times; each result is taken and
    dropped as it completes (as a client would), then the server's stats."""
    t0 = time.perf_counter()
    left = [len(reqs)]
    errors = []
    finished = threading.Event()
    lock = threading.Lock()

    def consume(f):
        try:
            f.result()
        except Exception as e:  # reported below
            errors.append(e)
        with lock:
            left[0] -= 1
            if left[0] == 0:
                finished.set()

    for r in reqs:
        now = time.perf_counter() - t0
        if r["t"] > now:
            time.sleep(r["t"] - now)
        srv.submit(r["pairs"], region_bp=r["region_bp"], mean_only=r["mean_only"],
                   return_posterior=r["return_posterior"]).add_done_callback(consume)
    finished.wait()
    if errors:
        raise errors[0]
    return srv.stats(reset=True)


def run_served(dev, rates=(10, 100, 1000, 2000), seconds=2.0, burst=300):
    """Serving stream over the resident small cohort (40 haplotypes, 2,127
    sites over 1 Mb): Poisson arrivals (seed 6), pair subsets log-uniform in
    [1, 8192] (clamped to the 780 pairs), regions log-uniform in [1 kb, 5 Mb]
    (clamped to the 1 Mb sequence), 20% full posterior.  Reports p50/p99
    latency per rate for the served loop and for the plain per-call path
    (FIFO, one call per query), and aggregate throughput of a burst of
    queries submitted at once."""
    from gamma_smc_cu_b200 import _core, synthetic
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    from gamma_smc_cu_b200.serve import TmrcaServer
    G, pos = synthetic.cohort("small")
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    ctx = _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
    out = {"workload": "small cohort 40 haps x 2,127 sites (1 Mb); queries: pairs log-uniform "
                       "[1, 8192] clamped to 780, regions log-uniform [1 kb, 5 Mb] clamped to "
                       "1 Mb, 20% full posterior", "rates": {}}
    with TmrcaServer(ctx, positions=pos, max_inflight=3, pinned_bytes=2 << 30) as srv:
        warm = synthetic.request_stream(pos, G.shape[0], 50, 0, seed=60)
        _served_latency(srv, warm)
        for r in warm[:10]:
            s0 = int(np.searchsorted(pos, r["region_bp"][0]))
            ctx.run_fb_window(r["pairs"], s0, s0 + 1)
        # aggregate throughput: every query submitted at once
        reqs = synthetic.request_stream(pos, G.shape[0], burst, 0, seed=6)
        st = _served_latency(srv, reqs)
        lat, ps, wall = _plain_latency(ctx, reqs, pos)
        out["burst"] = {"queries": burst, "served_pair_sites_per_s": st["pair_sites_per_s"],
                        "plain_pair_sites_per_s": ps / wall,
                        "speedup": st["pair_sites_per_s"] / (ps / wall),
                        "served_batches": st.get("batches")}
        for rate in rates:
            log(f"served rate {rate}/s")
            n = int(max(20, min(1000, rate * seconds)))
            reqs = synthetic.request_stream(pos, G.shape[0], n, rate, seed=6)
            st = _served_latency(srv, reqs)
            lat, ps, wall = _plain_latency(ctx, reqs, pos)
            out["rates"][str(rate)] = {
                "queries": n, "served_p50_ms": st["p50_ms"], "served_p99_ms": st["p99_ms"],
                "served_queue_p99_ms": st["queue_p99_ms"],
                "served_service_p99_ms": st["service_p99_ms"],
                "served_pair_sites_per_s": st["pair_sites_per_s"],
                "served_batches": st.get("batches"),
                "served_max_ms": st.get("max_ms"),
                "served_gc_pauses": st.get("gc_pauses"), "served_gc_max_ms": st.get("gc_max_ms"),
                "served_loop_stalls_ms": st.get("loop_stalls_ms"),
                "served_waits": {k: st.get(k, 0) for k in ("wait_executor", "wait_hbm",
                                                            "wait_arena", "outside_arena",
                                                            "redone_whole")},
                "plain_p50_ms": float(np.percentile(lat, 50) * 1e3),
                "plain_p99_ms": float(np.percentile(lat, 99) * 1e3),
                "plain_pair_sites_per_s": ps / wall}
    ctx.close()
    return out


def run_stream_stress(core=8192, flank=2048):
    """Large-cohort stress: 2,000 haplotypes x 200,000 sites (seeds 7/8),
    1,000,000 random pairs (seed 9), blockwise mean-only streamed to the host
    through pinned buffers (2e11 posteriors, 800 GB -- beyond host memory, so
    the sink checks and drops each unit).  Reports the delivered pair-sites/s
    (wall clock: context + all units on the host) and the scan kernels' own
    throughput from CUDA events."""
    import ctypes
    from gamma_smc_cu_b200 import _core, _lib, synthetic
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    t0 = time.perf_counter()
    G, pos = synthetic.cohort("cohort")
    pairs = synthetic.random_pairs(G.shape[0], 1_000_000, 9)
    gen_s = time.perf_counter() - t0
    S, P = G.shape[1], len(pairs)
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    L = _lib.load()
    stats = {"units": 0, "bytes": 0, "bad": 0}
    # parity sample: 16 of the million pairs, every site, collected from the
    # streamed units and checked against the oracle afterwards
    pick = np.sort(np.random.default_rng(13).choice(P, size=16, replace=False))
    kept = np.full((S, len(pick)), np.nan, np.float32)

    def sink(s0, s1, p0, p1, outs):
        m = outs["mean"]
        stats["units"] += 1
        stats["bytes"] += m.shape[0] * m.shape[1] * 4
        probe = m[:: max(1, m.shape[0] // 4), :: max(1, m.shape[1] // 8)]
        stats["bad"] += int((~np.isfinite(probe) | (probe <= 0)).sum())
        sel = np.nonzero((pick >= p0) & (pick < p1))[0]
        if sel.size:
            kept[s0:s1, sel] = m[:, pick[sel] - p0]
        return False

    t0 = time.perf_counter()
    ctx = _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
    _lib.check(L.gsmc_ctx_timing(ctx.handle, 1))
    ctx.run_fb_blockwise_stream(pairs, sink, core_block_sites=core, flank_sites=flank)
    wall = time.perf_counter() - t0
    kms = ctypes.c_double()
    launches = ctypes.c_int64()
    psites = ctypes.c_double()
    _lib.check(L.gsmc_ctx_timing_read(ctx.handle, ctypes.byref(kms), ctypes.byref(launches),
                                      ctypes.byref(psites)))
    ctx.close()
    parity = oracle_parity(G, pos, pairs[pick], mu, rho, core, flank, {"mean": kept})
    total = float(S) * P
    return {"parity": parity,
            "workload": "cohort 2,000 haps x 200,000 sites x 1,000,000 random pairs, blockwise "
                        f"core {core} / flank {flank}, mean_only, streamed to a host sink",
            "pair_sites": total, "seconds": wall, "value": total / wall, "unit": UNIT,
            "d2h_gb_per_s": stats["bytes"] / wall / 1e9, "units": stats["units"],
            "bad_samples": stats["bad"], "kernel_seconds": kms.value / 1e3,
            "kernel_pair_sites_per_s": psites.value / (kms.value / 1e3),
            "gpu_launches": int(launches.value), "data_generation_seconds": gen_s}


def run_e2e(G, pos, pairs, core, flank, steps):
    """Public API with host buffers: context (H2D genotypes and positions),
    blockwise run, D2H of every posterior into host arrays.  Timed with the
    results in page-locked buffers that the DMA writes directly
    (set_result_memory("pinned"); the buffers and the scan tables are made by
    an untimed first call and reused by the timed ones, as a repeated caller
    sees them), and once more into fresh pageable numpy arrays."""
    import psutil
    from gamma_smc_cu_b200 import _core, _lib
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    S, P = G.shape[1], len(pairs)
    avail = psutil.virtual_memory().available
    sites = S
    if 4.0 * S * P > 0.45 * avail:
        sites = int(0.45 * avail / (4.0 * P))
    Gs, ps = np.ascontiguousarray(G[:, :sites]), np.ascontiguousarray(pos[:sites])
    mu, rho = _estimate_scaled_params(Gs, ps, 1.25e-8, 1e-8, 1e4)
    plist = [tuple(p) for p in pairs.tolist()]

    def once():
        t0 = time.perf_counter()
        ctx = _core.FlowContext(Gs, ps, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0)
        t_ctx = time.perf_counter() - t0
        info = ctx.tables_info()
        r = ctx.run_fb_blockwise(plist, core_block_sites=core, flank_sites=flank,
                                 pair_batch_size=P, max_streams=1, mean_only=True)
        ctx.close()
        return r, info, t_ctx

    def infer_once():
        # the reference's own public entry point on the same inputs: input
        # checks, segregating-site filter, theta estimate on the GPU, context,
        # decode, results
        from gamma_smc_cu_b200.infer import infer_blockwise
        t0 = time.perf_counter()
        r = infer_blockwise(Gs, ps, pairs=plist, core_block_sites=core, flank_sites=flank,
                            pair_batch_size=P, mean_only=True)
        dt = time.perf_counter() - t0
        log(f"e2e through infer_blockwise {dt:.2f} s")
        del r
        return dt

    memory = "page-locked buffers reused across calls"
    api_s = None
    prev = _core.set_result_memory("pinned")
    try:
        t0 = time.perf_counter()
        r, info0, _ = once()   # builds the tables and the page-locked result buffer
        first_s = time.perf_counter() - t0
        log(f"e2e first call (page-locked results) {first_s:.1f} s")
        del r
        times, ctx_s = [], []
        for _ in range(max(1, steps)):
            t0 = time.perf_counter()
            r, info, t_ctx = once()
            times.append(time.perf_counter() - t0)
            ctx_s.append(t_ctx)
            log(f"e2e step {times[-1]:.2f} s")
            del r
        api_s = infer_once()
    except MemoryError as e:   # the host could not page-lock the results
        memory = f"pageable numpy arrays (page-locking failed: {e})"
        times = None
    finally:
        _core.set_result_memory(prev)
        _lib.check(_lib.load().gsmc_host_cache_limit(0))        # give the memory back
        _lib.check(_lib.load().gsmc_host_cache_limit(256 << 30))
    if times is None:
        times, ctx_s = [], []
        r, info0, _ = once()
        first_s = 0.0
        del r
        for _ in range(max(1, steps)):
            t0 = time.perf_counter()
            r, info, t_ctx = once()
            times.append(time.perf_counter() - t0)
            ctx_s.append(t_ctx)
            del r
    log("e2e pageable step")
    t0 = time.perf_counter()
    r, _, _ = once()
    pageable_s = time.perf_counter() - t0
    del r
    t = float(np.mean(times))
    return {"value": P * sites / t, "unit": UNIT,
            "h2d_bytes_per_step": int(Gs.nbytes + ps.nbytes + 8 * P),
            "d2h_bytes_per_step": int(4 * sites * P), "seconds_per_step": t, "sites": sites,
            "steps": len(times), "result_memory": memory,
            "context_seconds_per_step": float(np.mean(ctx_s)),
            "first_call_seconds": first_s,
            "table_build_seconds_first_call": info0["build_seconds"],
            "tables_reused_in_timed_steps": bool(info["reused"]),
            "pageable_seconds": pageable_s, "pageable_value": P * sites / pageable_s,
            "infer_blockwise_seconds": api_s}


# ------------------------------------------------------------ profiling cases
# Small, self-contained runs of each kernel for profilers (`--case NAME
# [--repeat N]`): each builds its inputs, runs once to warm up and then
# `--repeat` more times.  Inputs/outputs stay above the 126 MB L2 (so DRAM
# counters mean something) while the device holds a few GB at most.
#   scan      cached FB, chromosome cohort, 8,192 sites x 63,190 pairs,
#             blockwise core 512 / flank 128 (16 windows x 247 tiles of 256
#             pairs: the two-pairs-per-thread shape of the full job), mean-only
#   full      cached FB, mean + alpha + beta, 4,096 sites x 63,190 pairs,
#             blockwise core 256 / flank 64 (16 windows, two pairs per thread)
#   full_slice  cached FB, mean + alpha + beta, one 50,000-site window x 8,192
#             pairs in exact speculative chunks (the full-posterior slice's
#             shape), two pairs per thread
#   batch     64 uneven jobs (1-2,000 pairs, 2k-40k-site windows) over a
#             60,000-site slice, one executor launch (32-thread tiles,
#             4,096-site chunks)
#   summary   per-site summary, all 63,190 pairs x 20,000 sites (2,048 / 1,024)
#   fwd       forward-only posterior, 8,192 pairs x 20,000 sites
#   uncached  uncached flow-field FB, 4,096 pairs x 10,000 sites
#   flowgen   GPU flow-field generation, 51 x 50 cells, constant Ne
#   fwd_spec  forward-only posterior, 2,000 pairs x 400,000 sites (exact
#             speculative site chunks)
#   uncached_spec  uncached flow-field FB, 500 pairs x 200,000 sites (same)

def _case_ctx(n_sites):
    from gamma_smc_cu_b200 import _core, synthetic
    from gamma_smc_cu_b200.infer import _estimate_scaled_params
    G, pos = synthetic.cohort("chrom", n_sites=n_sites)
    mu, rho = _estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    return _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0), G, pos


def case_scan(repeat):
    import torch
    from gamma_smc_cu_b200 import _lib, synthetic
    ctx, G, pos = _case_ctx(8192)
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
    from gamma_smc_cu_b200 import _lib, synthetic
    ctx, G, pos = _case_ctx(4096)
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


def case_full_slice(repeat):
    """The full-posterior slice's shape at 8,192 pairs: one 50,000-site window
    (core = the whole slice, flank 2,048), mean + alpha + beta, exact
    speculative chunks with 2,048-site burn-ins, two pairs per thread."""
    import torch
    from gamma_smc_cu_b200 import _lib, synthetic
    os.environ["GSMC_PAIRS_PER_THREAD"] = "2"
    ctx, G, pos = _case_ctx(50000)
    pairs = synthetic.random_pairs(G.shape[0], 8192, 31)
    dev = torch.device("cuda", ctx.device_id)
    pi = torch.from_numpy(np.ascontiguousarray(pairs[:, 0])).to(dev)
    pj = torch.from_numpy(np.ascontiguousarray(pairs[:, 1])).to(dev)
    S, P = G.shape[1], len(pairs)
    outs = [torch.empty((S, P), device=dev) for _ in range(3)]
    L = _lib.load()
    for _ in range(1 + repeat):
        _lib.check(L.gsmc_run_fb_blockwise_device(
            ctx.handle, pi.data_ptr(), pj.data_ptr(), P, S, 2048, _lib.GSMC_POSTERIOR,
            outs[0].data_ptr(), None, None, outs[1].data_ptr(), outs[2].data_ptr(), P, 0, None))
    torch.cuda.synchronize()
    print("scan shape", ctx.scan_shape(), "speculative", ctx.spec_stats())


def case_batch(repeat):
    import torch
    from gamma_smc_cu_b200.batch import DeviceBatch, Executor, Job, Layout, _count_tasks
    from gamma_smc_cu_b200 import synthetic
    ctx, G, pos = _case_ctx(60000)
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
    from gamma_smc_cu_b200 import synthetic
    # enough (window, pair tile) tasks to fill the GPU twice, so the call runs
    # the summary instantiation itself (fewer go through per-pair means in
    # speculative chunks)
    ctx, G, pos = _case_ctx(20000)
    pairs = synthetic.all_pairs(G.shape[0])
    for _ in range(1 + repeat):
        ctx.run_fb_summary(pairs, core_block_sites=2048, flank_sites=1024)


def case_fwd(repeat):
    from gamma_smc_cu_b200 import synthetic
    ctx, G, pos = _case_ctx(20000)
    pairs = synthetic.random_pairs(G.shape[0], 8192, 4)
    for _ in range(1 + repeat):
        ctx.run_fwd(pairs)


def case_uncached(repeat):
    from gamma_smc_cu_b200 import _core, synthetic
    G, pos = synthetic.cohort("chrom", n_sites=10000)
    pairs = synthetic.random_pairs(G.shape[0], 4096, 6)
    for _ in range(1 + repeat):
        _core.gamma_smc_flow_fb(G, pos, pairs, mean_only=True)


def case_flowgen(repeat):
    from gamma_smc_cu_b200.demographic import generate_flow_field
    for _ in range(1 + repeat):
        generate_flow_field(verbose=False)


def case_fwd_spec(repeat):
    from gamma_smc_cu_b200 import synthetic
    ctx, G, pos = _case_ctx(400000)
    pairs = synthetic.random_pairs(G.shape[0], 2000, 4)
    for _ in range(1 + repeat):
        ctx.run_fwd(pairs)


def case_uncached_spec(repeat):
    from gamma_smc_cu_b200 import _core, synthetic
    G, pos = synthetic.cohort("chrom", n_sites=200000)
    pairs = synthetic.random_pairs(G.shape[0], 500, 4)
    for _ in range(1 + repeat):
        _core.gamma_smc_flow_fb(G, pos, pairs, mean_only=True)


CASES = {"scan": case_scan, "full": case_full, "full_slice": case_full_slice, "batch": case_batch,
         "summary": case_summary,
         "fwd": case_fwd, "uncached": case_uncached, "flowgen": case_flowgen,
         "fwd_spec": case_fwd_spec, "uncached_spec": case_uncached_spec}


if __name__ == "__main__":
    main()
