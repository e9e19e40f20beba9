"""Autotuner for batched scan launches.

Picks the executor configuration -- pair-tile width (threads per pair tile:
pairs per CTA), pairs per thread, and sites per chunk (``core_block_sites``
with a fixed ``flank_sites`` of burn-in) -- that runs a sample of a job mix
fastest on the current GPU, timing each candidate with CUDA events.  Results
are cached per (GPU, cohort shape, job-mix class) in a JSON file
(``$GSMC_AUTOTUNE_CACHE``, default ``~/.cache/gamma_smc_cu_b200/autotune.json``)
so a later process with the same class of work skips the search.

Chunking changes which sites a window's burn-in starts from; with the
default 2,048-site flank the chunked posteriors equal the whole-window ones
to float32 precision on realistic data (the tests check the 1e-4 bound).
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from .batch import DeviceBatch, Executor, Layout, _count_tasks

CHUNKS = (0, 4096, 8192, 16384, 32768)
SHAPES = ((128, 1), (128, 2), (32, 1), (32, 2))


def _bucket(x):
    return int(round(math.log2(max(1.0, float(x)))))


def job_class(jobs):
    """Coarse signature of a job mix: log2 buckets of its size statistics."""
    pairs = np.array([j.n_pairs for j in jobs] or [0])
    rows = np.array([j.rows for j in jobs] or [0])
    post = np.mean([not j.mean_only or j.return_posterior for j in jobs]) if jobs else 0.0
    return (f"n{_bucket(len(jobs))}-p{_bucket(np.median(pairs))}-P{_bucket(pairs.max())}"
            f"-w{_bucket(np.median(rows))}-W{_bucket(rows.max())}-f{int(round(post * 4))}")


def _cache_path():
    return os.environ.get("GSMC_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "gamma_smc_cu_b200", "autotune.json")


def _load_cache():
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(cache):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def cache_key(ctx, jobs):
    import torch
    name = torch.cuda.get_device_name(ctx.device_id)
    return f"{name}|haps{ctx.n_haps}|sites{_bucket(ctx.n_sites)}|{job_class(jobs)}"


def time_config(ctx, jobs, config, repeats=2, stream=None):
    """Mean device milliseconds of one batched launch of ``jobs`` under
    ``config`` (after one warm-up run)."""
    import torch
    dev = torch.device("cuda", ctx.device_id)
    cfg = dict(config)
    cfg.setdefault("max_tasks", max(1 << 10, _count_tasks(jobs, cfg)))
    if int(cfg.get("core_block_sites", 0)) <= 0:
        cfg.setdefault("max_window_sites", max([j.rows for j in jobs] + [1]))
    ex = Executor(ctx, **cfg)
    try:
        st = stream or torch.cuda.Stream(dev)
        b = DeviceBatch(Layout(jobs), dev)
        b.allocate(st)
        with torch.cuda.stream(st):
            b.d_pairs.copy_(b.h_pairs, non_blocking=True)
        run = lambda: ex.run(b.layout, b.d_pairs.data_ptr(), b.d_out.data_ptr(), st.cuda_stream)
        run()
        st.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(repeats):
            run()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / repeats
    finally:
        ex.close()


def autotune(ctx, jobs, flank_sites=2048, chunks=CHUNKS, shapes=SHAPES, use_cache=True,
             max_sample_jobs=512, verbose=False):
    """Best executor kwargs for ``jobs`` on ``ctx``'s GPU.

    Searches sites-per-chunk with the default launch shape, then launch
    shapes at the best chunk size.  Returns a dict of Executor kwargs plus
    ``"ms"`` (the best time) and ``"searched"`` (all timings)."""
    key = cache_key(ctx, jobs)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        return dict(cache[key], cached=True)
    sample = list(jobs)
    if len(sample) > max_sample_jobs:
        idx = np.random.default_rng(0).choice(len(sample), max_sample_jobs, replace=False)
        sample = [sample[i] for i in sorted(idx)]
    longest = max([j.rows for j in sample] + [1])
    searched = {}

    def trial(width, ppt, core):
        cfg = {"tile_width": width, "pairs_per_thread": ppt, "core_block_sites": core,
               "flank_sites": flank_sites}
        k = f"w{width}-np{ppt}-core{core}"
        try:
            searched[k] = time_config(ctx, sample, cfg)
        except (MemoryError, RuntimeError, ValueError) as e:  # e.g. pool does not fit
            searched[k] = float("inf")
            if verbose:
                print(f"[autotune] {k}: {e}", flush=True)
        if verbose:
            print(f"[autotune] {k}: {searched[k]:.3f} ms", flush=True)
        return searched[k]

    w0, p0 = shapes[0]
    best_core = min((c for c in chunks if c <= 0 or c < longest),
                    key=lambda c: trial(w0, p0, c))
    best_shape = min(shapes, key=lambda s: searched.get(f"w{s[0]}-np{s[1]}-core{best_core}")
                     if f"w{s[0]}-np{s[1]}-core{best_core}" in searched
                     else trial(s[0], s[1], best_core))
    best = {"tile_width": best_shape[0], "pairs_per_thread": best_shape[1],
            "core_block_sites": best_core, "flank_sites": flank_sites,
            "ms": searched[f"w{best_shape[0]}-np{best_shape[1]}-core{best_core}"],
            "searched": searched, "when": time.time()}
    if use_cache:
        cache = _load_cache()
        cache[key] = best
        _store_cache(cache)
    return dict(best, cached=False)


def executor_kwargs(tuned):
    """The Executor keyword arguments of an autotune result."""
    return {k: tuned[k] for k in ("tile_width", "pairs_per_thread", "core_block_sites",
                                  "flank_sites")}
