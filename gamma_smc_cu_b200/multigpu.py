"""Pair-parallel decoding over several GPUs.

Pairs are independent, so GPUs split them with no data-path exchange: every
device holds its own context (genotypes, tables) and decodes a contiguous
range of the pair list; full results are concatenated along the pair axis and
per-site summaries are merged as pair-weighted float64 sums.

* :class:`MultiGPUFlowContext` -- the reference's single-process API
  (python/gamma_smc_cu/multigpu.py:18-179): one FlowContext per device id, a
  persistent thread pool drives them concurrently (the library releases the
  GIL inside every call), results joined on the host.
* :class:`DistributedFlowContext` -- one process per GPU under
  ``torch.distributed`` (torchrun): each rank builds a context on its own
  device and decodes its shard; ``run_fb``/``run_fwd`` gather the shards to
  rank 0, ``run_fb_summary`` all-reduces the per-site sums, minima and maxima
  (3 x n_sites values) so every rank returns the same summary.

Both split pairs by the reference's rule (multigpu.py:59-70):
ceil(n_pairs / n_parts) pairs per part, trailing parts shorter or empty.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np


def split_pairs(n_pairs, n_parts):
    """(start, stop) of each part: ceil(n_pairs / n_parts) pairs per part."""
    n_pairs, n_parts = int(n_pairs), max(1, int(n_parts))
    chunk = -(-n_pairs // n_parts)
    return [(min(i * chunk, n_pairs), min((i + 1) * chunk, n_pairs)) for i in range(n_parts)]


def _as_pairs(pairs):
    p = np.asarray(pairs, dtype=np.int32)
    return p.reshape(-1, 2) if p.size else np.zeros((0, 2), np.int32)


def _empty(S, mean_only):
    d = {"mean": np.empty((S, 0), np.float32)}
    if not mean_only:
        d["lower"] = np.empty((S, 0), np.float32)
        d["upper"] = np.empty((S, 0), np.float32)
    return d


def _concat(results, S, mean_only):
    results = [r for r in results if r is not None]
    if not results:
        return _empty(S, mean_only)
    return {k: np.concatenate([r[k] for r in results], axis=1) for k in results[0]}


def _summary_part(ctx, pairs, chunk_size, S):
    """float64 sum over pairs of the site mean, and site extremes, over one
    part in chunks of ``chunk_size`` pairs (multigpu.py:80-91)."""
    site_sum = np.zeros(S, np.float64)
    lo = np.full(S, np.inf)
    hi = np.full(S, -np.inf)
    total = 0
    step = max(1, int(chunk_size))
    for i in range(0, len(pairs), step):
        chunk = pairs[i:i + step]
        r = ctx.run_fb_summary(chunk)
        site_sum += r["site_mean"].astype(np.float64) * len(chunk)
        lo = np.minimum(lo, r["site_min"])
        hi = np.maximum(hi, r["site_max"])
        total += len(chunk)
    return site_sum, lo, hi, total


def _summary_result(site_sum, lo, hi, total, n_gpus, S):
    if total == 0:
        return {"site_mean": np.zeros(S, np.float32), "n_pairs": 0, "n_gpus": 0}
    return {"site_mean": (site_sum / total).astype(np.float32),
            "site_min": np.asarray(lo, np.float32), "site_max": np.asarray(hi, np.float32),
            "n_pairs": int(total), "n_gpus": n_gpus}


def _default_factory(G, positions, Ne, mu, rho, flow_field_path, cache_steps):
    from ._core import FlowContext
    return FlowContext(G, positions, float(Ne), mu, rho, flow_field_path, cache_steps)


class MultiGPUFlowContext:
    """FlowContext work split across the devices ``gpu_ids`` (None = every
    visible device).  Same constructor and methods as the reference's
    MultiGPUFlowContext; ``context_factory`` (keyword only) replaces the
    per-device FlowContext constructor."""

    def __init__(self, G, positions, Ne, mu, rho, flow_field_path, gpu_ids=None,
                 cache_steps=0, *, context_factory=None):
        from . import _core
        factory = context_factory or _default_factory
        if gpu_ids is None:
            gpu_ids = list(range(_core.get_device_count()))
        self.gpu_ids = list(gpu_ids)
        if not self.gpu_ids:
            raise ValueError("MultiGPUFlowContext needs at least one device")
        self.n_gpus = len(self.gpu_ids)
        self.S = len(positions)
        self.contexts = []
        for gid in self.gpu_ids:
            if context_factory is None:
                _core.set_device(gid)
            self.contexts.append(factory(G, positions, Ne, mu, rho, flow_field_path,
                                         cache_steps))
        if context_factory is None:
            _core.set_device(self.gpu_ids[0])
        self._pool = ThreadPoolExecutor(max_workers=self.n_gpus)

    def __del__(self):
        pool = getattr(self, "_pool", None)
        if pool is not None:
            pool.shutdown(wait=False)

    def _split_pairs(self, pairs):
        """Per-device pair chunks (the reference's split)."""
        pairs = _as_pairs(pairs)
        return [pairs[a:b] for a, b in split_pairs(len(pairs), self.n_gpus)]

    def _map(self, fn, pairs):
        parts = self._split_pairs(pairs)
        futures = [self._pool.submit(fn, self.contexts[i], p) if len(p) else None
                   for i, p in enumerate(parts)]
        return [f.result() if f is not None else None for f in futures]

    def run_fb_summary(self, pairs, chunk_size=10000):
        """Per-site mean over every pair (float64 pair-weighted merge of the
        per-chunk summaries), plus site_min / site_max."""
        if len(pairs) == 0:
            return _summary_result(None, None, None, 0, 0, self.S)
        parts = self._map(lambda c, p: _summary_part(c, p, chunk_size, self.S), pairs)
        parts = [p for p in parts if p is not None]
        return _summary_result(sum(p[0] for p in parts),
                               np.minimum.reduce([p[1] for p in parts]),
                               np.maximum.reduce([p[2] for p in parts]),
                               sum(p[3] for p in parts), self.n_gpus, self.S)

    def run_fwd(self, pairs, mean_only=True):
        """Forward-only filtering; 'mean' [S, n_pairs] (+ 'lower'/'upper')."""
        if len(pairs) == 0:
            return _empty(self.S, mean_only)
        return _concat(self._map(lambda c, p: c.run_fwd(p, mean_only), pairs), self.S,
                       mean_only)

    def run_fb(self, pairs, mean_only=True):
        """Forward-backward smoothing; 'mean' [S, n_pairs] (+ 'lower'/'upper')."""
        if len(pairs) == 0:
            return _empty(self.S, mean_only)
        return _concat(self._map(lambda c, p: c.run_fb(p, mean_only), pairs), self.S,
                       mean_only)

    @property
    def device_ids(self):
        return self.gpu_ids

    def close(self):
        self._pool.shutdown(wait=True)
        for c in self.contexts:
            close = getattr(c, "close", None)
            if close is not None:
                close()


class DistributedFlowContext:
    """One process per GPU under an initialised ``torch.distributed`` group:
    every rank builds its context (``context_factory``, default FlowContext
    on the current device) and decodes ``split_pairs(n, world)[rank]``."""

    def __init__(self, G, positions, Ne, mu, rho, flow_field_path, cache_steps=0, *,
                 group=None, context_factory=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.S = len(positions)
        self.ctx = (context_factory or _default_factory)(G, positions, Ne, mu, rho,
                                                         flow_field_path, cache_steps)

    def shard(self, n_pairs):
        """(start, stop) of this rank's pairs."""
        return split_pairs(n_pairs, self.world)[self.rank]

    def _gather(self, local, gather):
        import torch.distributed as dist
        if not gather:
            return local
        parts = [None] * self.world if self.rank == 0 else None
        dist.gather_object(local, parts, dst=0, group=self.group)
        return parts

    def _run(self, method, pairs, mean_only, gather):
        pairs = _as_pairs(pairs)
        a, b = self.shard(len(pairs))
        local = getattr(self.ctx, method)(pairs[a:b], mean_only) if b > a else None
        parts = self._gather(local, gather)
        if not gather:
            return local if local is not None else _empty(self.S, mean_only)
        return _concat(parts, self.S, mean_only) if self.rank == 0 else None

    def run_fb(self, pairs, mean_only=True, gather=True):
        """Forward-backward over all pairs: rank 0 gets [S, n_pairs] arrays
        (other ranks None); ``gather=False`` returns this rank's shard."""
        return self._run("run_fb", pairs, mean_only, gather)

    def run_fwd(self, pairs, mean_only=True, gather=True):
        """Forward-only filtering, sharded like :meth:`run_fb`."""
        return self._run("run_fwd", pairs, mean_only, gather)

    def run_fb_summary(self, pairs, chunk_size=10000):
        """Per-site summary over all pairs, the same on every rank: float64
        sums, minima and maxima are all-reduced (on the GPU under NCCL)."""
        import torch
        import torch.distributed as dist
        pairs = _as_pairs(pairs)
        a, b = self.shard(len(pairs))
        s, lo, hi, n = _summary_part(self.ctx, pairs[a:b], chunk_size, self.S)
        if dist.get_backend(self.group) == "nccl":
            dev = torch.device("cuda", torch.cuda.current_device())
        else:
            dev = torch.device("cpu")
        t = [torch.from_numpy(x).to(dev) for x in (s, lo, hi)]
        dist.all_reduce(t[0], op=dist.ReduceOp.SUM, group=self.group)
        dist.all_reduce(t[1], op=dist.ReduceOp.MIN, group=self.group)
        dist.all_reduce(t[2], op=dist.ReduceOp.MAX, group=self.group)
        s, lo, hi = (x.cpu().numpy() for x in t)
        return _summary_result(s, lo, hi, len(pairs), self.world, self.S)

    def close(self):
        close = getattr(self.ctx, "close", None)
        if close is not None:
            close()
