"""Continuous-batching TMRCA query server over one resident context.

A query asks for the posterior of a pair subset over a region (a site range,
or a base-pair range mapped to sites through the positions) and gets back the
same result dict ``FlowContext.run_fb_window`` returns for it.  Queries arrive
at any time from any thread (``submit`` returns a ``concurrent.futures.Future``).

The scheduler thread keeps several batches in flight, each on its own
executor (its own forward-state pool and task list) and CUDA stream.  As soon
as an executor is free it admits every waiting query that fits -- into the
device-memory budget for outputs (free HBM measured at start-up, minus
headroom) and the batch's task capacity -- and launches them together as one
persistent kernel, followed by the device-to-host copy of their outputs on
the same stream.  Queries that arrive while earlier batches are on the GPU
therefore start as soon as an executor and memory free up, and their work
overlaps the tail of the running batches on the device.  Genotypes, gap codes
and flow-field tables stay resident in the context the whole time.

A query whose outputs alone exceed the whole budget is rejected with
MemoryError; malformed queries are rejected at ``submit`` with ValueError.
``stats()`` reports latency percentiles (arrival to result), throughput and
admission counters.
"""
from __future__ import annotations

import collections
import gc
import threading
import time
import weakref
from concurrent.futures import Future

import numpy as np

from .batch import DeviceBatch, Executor, Job, Layout, _count_tasks, validate

BYTES_PER_FLOAT = 4


def _new_stream(device):
    import torch
    return torch.cuda.Stream(device)


def _free_device_bytes(device):
    import torch
    return torch.cuda.mem_get_info(device)[0]


def _prewarm(device, streams, device_bytes, pinned_bytes):
    """Fill the allocator caches a batch draws on, before serving starts.

    A batch's device buffers come from torch's caching allocator on its slot's
    stream, and cached blocks are kept per stream, so a slot's first batch of
    a new size calls cudaMalloc -- and, with little free memory, releases the
    cache with cudaFree, which waits for the device: milliseconds inside the
    scheduler loop.  One block of ``device_bytes`` per stream, freed at once,
    stays cached for that stream and is split for later batches.  Pinned
    staging of pair indices (torch's caching host allocator, power-of-two
    size classes) is warmed up to ``pinned_bytes`` the same way."""
    import torch
    for st in streams:
        with torch.cuda.stream(st):
            t = torch.empty(max(int(device_bytes), 1), dtype=torch.uint8, device=device)
        del t
    n = 4096
    while n <= max(int(pinned_bytes), 4096):
        t = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        del t
        n *= 2
    torch.cuda.synchronize(device)


def _new_arena(nbytes):
    return PinnedArena(nbytes)


def _bind_thread(device):
    import torch
    if torch.cuda.is_available():
        torch.cuda.set_device(device)


class _Region:
    """Owner of one arena region; numpy views of it keep it alive, and the
    region returns to the arena when the last view is garbage-collected."""

    def __init__(self, arena, offset, nbytes):
        self.__array_interface__ = {"shape": (nbytes // BYTES_PER_FLOAT,), "typestr": "<f4",
                                    "data": (arena.base + offset, False), "version": 3}
        weakref.finalize(self, arena.release, offset, nbytes)


class PinnedArena:
    """First-fit allocator over one pinned host buffer that results are
    copied into; hands out float32 views (see _Region)."""

    ALIGN = 256

    def __init__(self, nbytes):
        import torch
        self.size = int(nbytes)
        self._t = torch.empty(max(self.size, 1), dtype=torch.uint8, pin_memory=True)
        self.base = self._t.data_ptr()
        self._free = [(0, self.size)]   # sorted (offset, length)
        self._lock = threading.Lock()
        self.in_use = 0

    def alloc(self, nbytes):
        """A float32 view of nbytes (rounded up), or None if nothing fits."""
        n = -(-max(int(nbytes), 1) // self.ALIGN) * self.ALIGN
        with self._lock:
            for i, (off, ln) in enumerate(self._free):
                if ln >= n:
                    if ln == n:
                        del self._free[i]
                    else:
                        self._free[i] = (off + n, ln - n)
                    self.in_use += n
                    break
            else:
                return None
        return np.asarray(_Region(self, off, n))

    def largest_free(self):
        """Bytes of the largest free block (the biggest alloc that succeeds)."""
        with self._lock:
            return max((ln for _, ln in self._free), default=0)

    def release(self, off, n):
        with self._lock:
            self.in_use -= n
            self._free.append((off, n))
            self._free.sort()
            merged = []
            for o, ln in self._free:
                if merged and merged[-1][0] + merged[-1][1] == o:
                    merged[-1] = (merged[-1][0], merged[-1][1] + ln)
                else:
                    merged.append((o, ln))
            self._free = merged


def _pinned_floats(n):
    """A pinned float32 array of n elements outside the arena (torch's
    caching host allocator)."""
    import torch
    return torch.empty(max(int(n), 1), dtype=torch.float32, pin_memory=True).numpy()


class _Request:
    __slots__ = ("job", "future", "t_arrive", "t_admit", "t_done", "bytes", "tasks")

    def __init__(self, job, future, t_arrive, nbytes, tasks):
        self.job = job
        self.future = future
        self.t_arrive = t_arrive
        self.t_admit = None
        self.t_done = None
        self.bytes = nbytes
        self.tasks = tasks


class _Slot:
    """One executor, its stream, and the batch it is running (if any)."""

    def __init__(self, executor, stream):
        self.executor = executor
        self.stream = stream
        self.batch = None
        self.requests = []
        self.bytes = 0


class TmrcaServer:
    """Request loop with continuous batching over ``ctx`` (a FlowContext).

    ``positions`` (site coordinates) enables base-pair regions.
    ``max_inflight`` executors run concurrently; ``core_block_sites`` /
    ``flank_sites`` chunk long windows (0 = whole windows), ``tile_width`` /
    ``pairs_per_thread`` set the launch shape (see :mod:`.tune` for picking
    them); ``hbm_budget`` bounds the device bytes of in-flight outputs
    (default: half the free device memory after the executors exist).
    """

    def __init__(self, ctx, positions=None, max_inflight=3, core_block_sites=4096,
                 flank_sites=2048, tile_width=128, pairs_per_thread=1, use_graph=True,
                 hbm_budget=None, max_tasks=1 << 15, max_batch_requests=4096,
                 max_batch_pair_sites=1 << 29, pinned_bytes=1 << 30, poll_interval=50e-6,
                 freeze_gc=True):
        self.ctx = ctx
        self.positions = None if positions is None else np.asarray(positions, np.float64)
        self.device = ctx.device_id
        self.config = {"tile_width": tile_width, "pairs_per_thread": pairs_per_thread,
                       "core_block_sites": core_block_sites, "flank_sites": flank_sites,
                       "use_graph": use_graph, "max_tasks": max_tasks}
        if core_block_sites <= 0:
            self.config["max_window_sites"] = ctx.n_sites
        # looked up on the module at call time, so host-side tests can
        # substitute fakes for the device pieces
        self.slots = [_Slot(Executor(ctx, **self.config), _new_stream(self.device))
                      for _ in range(max(1, int(max_inflight)))]
        if hbm_budget is None:
            hbm_budget = int(0.5 * _free_device_bytes(self.device))
        self.hbm_budget = int(hbm_budget)
        self.max_tasks = int(max_tasks)
        self.max_batch_requests = int(max_batch_requests)
        self.max_batch_pair_sites = float(max_batch_pair_sites)
        self.arena = _new_arena(pinned_bytes) if pinned_bytes else None
        # a batch's outputs fit the largest arena block (or wait for one)
        _prewarm(self.device, [sl.stream for sl in self.slots],
                 min(self.hbm_budget, int(pinned_bytes) if pinned_bytes else 1 << 28),
                 min(8 * self.max_tasks * 128, 8 << 20))
        self.poll_interval = float(poll_interval)
        self._pending = collections.deque()
        self._cv = threading.Condition()
        self._closing = False
        self._in_use = 0
        self._done = []           # finished requests (for stats)
        self.counters = collections.Counter()
        self._redo_ex = None
        self._redo_tasks = 0
        self._redo_stream = None
        # Diagnostics of the latency tail: the longest scheduler-loop stalls
        # (what the loop was doing), and the cyclic garbage collector's pauses
        # while serving (they stop the scheduler thread too).
        self._stalls = []          # (ms, what)
        self._admit_step = ""
        self._gc_pauses = []       # (generation, ms)
        self._gc_t0 = None
        if freeze_gc:
            # A full collection traverses every tracked object of the process
            # (with torch loaded: hundreds of thousands, ~0.1 s).  Objects that
            # exist when the server starts are long-lived, so move them out of
            # the collector's generations; collections while serving then
            # traverse only what was made since.  Process-wide, as Python's
            # gc.freeze is.
            gc.collect()
            gc.freeze()
        gc.callbacks.append(self._on_gc)
        self._thread = threading.Thread(target=self._loop, name="gsmc-serve", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------ client API

    def sites_of(self, start_bp, end_bp):
        """Site range [s0, s1) of the sites with start_bp <= position < end_bp."""
        if self.positions is None:
            raise ValueError("the server has no positions; give site ranges")
        s0 = int(np.searchsorted(self.positions, start_bp, side="left"))
        s1 = int(np.searchsorted(self.positions, end_bp, side="left"))
        return s0, max(s0, s1)

    def submit(self, pairs, site_begin=None, site_end=None, region_bp=None, mean_only=True,
               return_posterior=False):
        """Queue one query; returns a Future of its result dict."""
        if region_bp is not None:
            site_begin, site_end = self.sites_of(*region_bp)
        if site_begin is None:
            site_begin = 0
        if site_end is None:
            site_end = self.ctx.n_sites
        job = Job(pairs, site_begin, site_end, mean_only=mean_only,
                  return_posterior=return_posterior)
        validate(job, self.ctx.n_haps, self.ctx.n_sites)
        fut = Future()
        req = _Request(job, fut, time.perf_counter(), job.layout_floats * BYTES_PER_FLOAT,
                       _count_tasks([job], self.config))
        with self._cv:
            if self._closing:
                raise RuntimeError("server is closed")
            self._pending.append(req)
            self.counters["submitted"] += 1
            self._cv.notify()
        return fut

    def _on_gc(self, phase, info):
        if phase == "start":
            self._gc_t0 = time.perf_counter()
        elif self._gc_t0 is not None:
            ms = (time.perf_counter() - self._gc_t0) * 1e3
            self._gc_t0 = None
            if ms >= 1.0 and len(self._gc_pauses) < 10000:
                self._gc_pauses.append((int(info.get("generation", -1)), ms))

    def _note_stall(self, t0, what):
        ms = (time.perf_counter() - t0) * 1e3
        if ms >= 2.0 and len(self._stalls) < 10000:
            self._stalls.append((ms, what))

    def close(self, wait=True):
        with self._cv:
            self._closing = True
            self._cv.notify()
        if wait:
            self._thread.join()
        try:
            gc.callbacks.remove(self._on_gc)
        except ValueError:
            pass
        for s in self.slots:
            s.executor.close()
        if self._redo_ex is not None:
            self._redo_ex.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stats(self, reset=False):
        """Latency percentiles (ms), throughput and counters of finished queries."""
        with self._cv:
            done = list(self._done)
            counters = dict(self.counters)
            stalls, pauses = list(self._stalls), list(self._gc_pauses)
            if reset:
                self._done.clear()
                self.counters.clear()
                self._stalls.clear()
                self._gc_pauses.clear()
        out = {"completed": len(done), **counters}
        # longest scheduler stalls and collector pauses (>= 2 ms / >= 1 ms)
        out["loop_stalls_ms"] = [(round(ms, 2), what) for ms, what in sorted(stalls)[-5:][::-1]]
        out["gc_pauses"] = len(pauses)
        out["gc_max_ms"] = max((ms for _, ms in pauses), default=0.0)
        if done:
            t = np.array(done)
            lat = (t[:, 2] - t[:, 0]) * 1e3
            queue = (t[:, 1] - t[:, 0]) * 1e3
            service = (t[:, 2] - t[:, 1]) * 1e3
            span = float(t[:, 2].max() - t[:, 0].min())
            ps = float(t[:, 3].sum())
            out.update({"p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)),
                        "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
                        "queue_p50_ms": float(np.percentile(queue, 50)),
                        "queue_p99_ms": float(np.percentile(queue, 99)),
                        "service_p50_ms": float(np.percentile(service, 50)),
                        "service_p99_ms": float(np.percentile(service, 99)),
                        "pair_sites": ps, "span_s": span,
                        "pair_sites_per_s": ps / span if span > 0 else None})
        return out

    # ------------------------------------------------------------- scheduler

    def _redo_whole(self, job):
        """One query decoded as a single whole window (exact), on an executor
        made on first need: one-warp tiles, no chunking, a pool for at least
        one CTA of whole-window slots."""
        # one whole window in one-warp tiles of 32 pairs: ceil(n_pairs / 32)
        # tasks; the executor is sized for the largest redo so far
        need = max(1, -(-job.n_pairs // 32))
        if self._redo_ex is None or need > self._redo_tasks:
            if self._redo_ex is not None:
                self._redo_ex.close()
                self._redo_ex = None
            slot = 4 * max(1, self.ctx.n_sites) * 32 * 8   # 4 one-warp tiles, float2 states
            self._redo_tasks = max(1 << 8, need)
            self._redo_ex = Executor(self.ctx, tile_width=32, pairs_per_thread=1,
                                     core_block_sites=0, max_window_sites=self.ctx.n_sites,
                                     max_tasks=self._redo_tasks,
                                     max_pool_bytes=max(1 << 30, slot), use_graph=False)
            if self._redo_stream is None:
                self._redo_stream = _new_stream(self.device)
        b = DeviceBatch(Layout([job]), self.device)
        b.launch(self._redo_ex, self._redo_stream)
        return b.to_host()[0]

    def _finish(self, slot):
        # views into the batch's pinned host buffer: an arena region returns
        # to the arena once the caller drops the last result array using it
        # done already; queries whose chunks failed the device check are
        # decoded again whole on the server's own executor (never the context,
        # which callers may be using on other threads)
        try:
            results = slot.batch.results(redo=self._redo_whole)
        except Exception as e:  # a failed redo fails only its batch
            results = None
            for req in slot.requests:
                req.future.set_exception(e)
            with self._cv:
                self.counters["failed"] += len(slot.requests)
        now = time.perf_counter()
        for req, res in zip(slot.requests, results or []):
            req.t_done = now
            req.future.set_result(res)
        with self._cv:
            self._in_use -= slot.bytes
            # timings only: the requests (and the results their futures hold)
            # are not kept, so result memory returns once the caller drops it
            self._done.extend((r.t_arrive, r.t_admit, r.t_done, float(r.job.pair_sites))
                              for r in slot.requests if r.t_done is not None)
            self.counters["batches"] += 1
            if slot.batch.repaired:
                self.counters["redone_whole"] += slot.batch.repaired
        slot.batch = None
        slot.requests = []
        slot.bytes = 0

    def _admit(self, slot):
        """Move the waiting queries that fit into a new batch on ``slot``.

        A batch's results land in one block of the pinned arena, so it takes no
        more than the largest free block holds: allocating pinned memory
        outside the arena costs milliseconds to seconds.  A query larger than
        the free block waits while other batches are in flight (their results
        return to the arena as clients drop them); with none in flight, or if
        it exceeds the whole arena, it runs with its own pinned buffer."""
        take, nbytes, ntasks, work = [], 0, 0, 0.0
        cap = self.arena.largest_free() if self.arena is not None else None
        in_flight = any(s.batch is not None for s in self.slots)
        with self._cv:
            while self._pending and len(take) < self.max_batch_requests:
                req = self._pending[0]
                if req.bytes > self.hbm_budget or req.tasks > self.max_tasks:
                    self._pending.popleft()
                    self.counters["rejected"] += 1
                    req.future.set_exception(MemoryError(
                        f"query needs {req.bytes} bytes of outputs and {req.tasks} tasks; the "
                        f"server holds at most {self.hbm_budget} bytes and {self.max_tasks} "
                        "tasks per batch"))
                    continue
                if take and (self._in_use + nbytes + req.bytes > self.hbm_budget
                             or ntasks + req.tasks > self.max_tasks
                             or work + req.job.pair_sites > self.max_batch_pair_sites
                             or (cap is not None and nbytes + req.bytes > cap)):
                    break   # the batch is full; the rest go to the next free executor
                # why the head query waits (counted once per admission pass)
                if self._in_use + req.bytes > self.hbm_budget:
                    self.counters["wait_hbm"] += 1
                    break
                if (not take and cap is not None and req.bytes > cap and in_flight
                        and req.bytes <= self.arena.size):
                    self.counters["wait_arena"] += 1
                    break
                self._pending.popleft()
                take.append(req)
                nbytes += req.bytes
                ntasks += req.tasks
                work += req.job.pair_sites
            if not take:
                return False
            self._in_use += nbytes
            self.counters["admitted"] += len(take)
        now = time.perf_counter()
        for r in take:
            r.t_admit = now
        # the slowest step of this admission names a loop stall (_loop)
        steps = [now]
        try:
            layout = Layout([r.job for r in take])
            steps.append(time.perf_counter())
            host = self.arena.alloc(layout.out_floats * BYTES_PER_FLOAT) if self.arena else None
            if host is None:
                host = _pinned_floats(layout.out_floats)
                with self._cv:
                    self.counters["outside_arena"] += 1
            steps.append(time.perf_counter())
            batch = DeviceBatch(layout, self.device)
            steps.append(time.perf_counter())
            batch.launch(slot.executor, slot.stream, host=host)
            steps.append(time.perf_counter())
            names = ("layout", "host", "batch", "launch")
            d = [b - a for a, b in zip(steps, steps[1:])]
            self._admit_step = names[d.index(max(d))]
        except Exception as e:  # a launch failure fails the batch's queries
            with self._cv:
                self._in_use -= nbytes
                self.counters["failed"] += len(take)
            for r in take:
                r.future.set_exception(e)
            return True
        slot.batch, slot.requests, slot.bytes = batch, take, nbytes
        return True

    def _loop(self):
        _bind_thread(self.device)
        while True:
            busy = False
            for slot in self.slots:
                if slot.batch is not None and slot.batch.done.query():
                    t0 = time.perf_counter()
                    self._finish(slot)
                    self._note_stall(t0, "finish")
                    busy = True
            free = False
            for slot in self.slots:
                if slot.batch is None and self._pending:
                    free = True
                    t0 = time.perf_counter()
                    self._admit_step = "queue"
                    busy |= self._admit(slot)
                    self._note_stall(t0, "admit:" + self._admit_step)
            if self._pending and not free:
                self.counters["wait_executor"] += 1
            with self._cv:
                idle = all(s.batch is None for s in self.slots)
                if self._closing and not self._pending and idle:
                    return
                if not busy:
                    if idle and not self._pending:
                        self._cv.wait(timeout=0.05)
                    else:
                        self._cv.wait(timeout=self.poll_interval)
