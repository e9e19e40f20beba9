"""Batched scan jobs: many (pair set x site window) jobs in one persistent launch.

A :class:`Job` asks for the posterior of a set of haplotype pairs over a
window ``[site_begin, site_end)`` of a :class:`~gamma_smc_cu_b200.FlowContext`'s
sites.  Its result is what ``FlowContext.run_fb_window`` returns for the same
pairs and window: the window is decoded as one padded window of the
reference's block kernels (src/kernels/gamma_smc_flow.cu:632-669, 762-839).

An :class:`Executor` turns every job's window -- optionally cut into chunks of
``core_block_sites`` with ``flank_sites`` of burn-in, as ``run_fb_blockwise``
does for a chromosome -- and pair tiles into one device task list and runs it
as one persistent launch (``gsmc_exec_run``), optionally replayed as a CUDA
graph.  Each executor owns the scratch of one in-flight launch; the serving
loop (``serve.py``) keeps several in flight on separate streams.

torch provides the device buffers, pinned host buffers, streams and events;
the scan itself is the library's sm_100a kernel.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import GSMC_CI, GSMC_POSTERIOR, check

OUTPUT_KEYS = ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")


def _selected(mean_only, return_posterior):
    return [True, not mean_only, not mean_only, return_posterior, return_posterior]


@dataclass
class Job:
    """Posterior of ``pairs`` over sites ``[site_begin, site_end)``."""
    pairs: np.ndarray
    site_begin: int
    site_end: int
    mean_only: bool = True
    return_posterior: bool = False
    tag: object = field(default=None, compare=False)

    def __post_init__(self):
        p = np.asarray(self.pairs)
        if p.size == 0:
            p = p.reshape(0, 2)
        if p.ndim != 2 or p.shape[1] != 2:
            raise TypeError("pairs must be a sequence of (i, j) pairs")
        self.pairs = np.ascontiguousarray(p, dtype=np.int32)
        self.site_begin = int(self.site_begin)
        self.site_end = int(self.site_end)

    @property
    def n_pairs(self):
        return int(self.pairs.shape[0])

    @property
    def rows(self):
        return self.site_end - self.site_begin

    @property
    def flags(self):
        return (0 if self.mean_only else GSMC_CI) | (GSMC_POSTERIOR if self.return_posterior else 0)

    @property
    def n_outputs(self):
        return sum(_selected(self.mean_only, self.return_posterior))

    @property
    def output_floats(self):
        return self.rows * self.n_pairs * self.n_outputs

    @property
    def pair_sites(self):
        return self.rows * self.n_pairs


def validate(job, n_haps, n_sites):
    """Host-side checks of one job against a context (ValueError)."""
    if job.site_begin < 0 or job.site_end > n_sites or job.site_begin > job.site_end:
        raise ValueError(f"site window [{job.site_begin}, {job.site_end}) is out of range for "
                         f"{n_sites} sites")
    if job.n_pairs and (job.pairs.min() < 0 or job.pairs.max() >= n_haps):
        raise ValueError(f"pair index out of range for {n_haps} haplotypes")


class Layout:
    """Where each job's pairs and outputs sit in one flat batch buffer.

    Pairs: int32 ``[pi of job 0 | pj of job 0 | pi of job 1 | ...]``.
    Outputs: float32, per job its selected outputs in OUTPUT_KEYS order, each
    ``[rows, n_pairs]`` row-major, 64-float aligned.
    """

    def __init__(self, jobs):
        self.jobs = list(jobs)
        self.pair_off = []
        self.out_off = []
        po = 0
        oo = 0
        for j in self.jobs:
            self.pair_off.append(po)
            po += 2 * j.n_pairs
            offs = []
            for sel in _selected(j.mean_only, j.return_posterior):
                if sel:
                    offs.append(oo)
                    oo += -(-j.rows * j.n_pairs // 64) * 64
                else:
                    offs.append(None)
            self.out_off.append(offs)
        self.pair_ints = po
        self.out_floats = oo

    def pack_pairs(self, dst):
        """Write every job's pairs into the int32 array ``dst``."""
        for j, o in zip(self.jobs, self.pair_off):
            n = j.n_pairs
            dst[o:o + n] = j.pairs[:, 0]
            dst[o + n:o + 2 * n] = j.pairs[:, 1]

    def c_jobs(self, pair_base, out_base):
        """ctypes gsmc_job array for device buffers at the given addresses."""
        arr = (_lib.Job * len(self.jobs))()
        for k, (j, po, offs) in enumerate(zip(self.jobs, self.pair_off, self.out_off)):
            c = arr[k]
            c.pair_i = pair_base + 4 * po
            c.pair_j = pair_base + 4 * (po + j.n_pairs)
            c.n_pairs = j.n_pairs
            c.site_begin = j.site_begin
            c.site_end = j.site_end
            c.flags = j.flags
            for i, o in enumerate(offs):
                c.out[i] = None if o is None else out_base + 4 * o
            c.ld_out = j.n_pairs
            c.out_col0 = 0
        return arr

    def results(self, host):
        """Per-job result dicts of views into the float32 host array."""
        res = []
        for j, offs in zip(self.jobs, self.out_off):
            d = {}
            for key, o in zip(OUTPUT_KEYS, offs):
                if o is not None:
                    d[key] = host[o:o + j.rows * j.n_pairs].reshape(j.rows, j.n_pairs)
            res.append(d)
        return res


class Executor:
    """Scratch and launch machinery of one in-flight batch (``gsmc_exec``).

    ``tile_width`` (32 or 128 threads per pair tile) and ``pairs_per_thread``
    (1 or 2) set the launch shape; ``core_block_sites`` (<= 0: whole windows)
    and ``flank_sites`` set how job windows are chunked; ``max_window_sites``
    bounds a whole window when not chunking; ``use_graph`` replays upload and
    launch as one CUDA graph.
    """

    def __init__(self, ctx, tile_width=32, pairs_per_thread=1, core_block_sites=0,
                 flank_sites=2048, max_window_sites=0, max_tasks=1 << 16, max_pool_bytes=0,
                 max_ctas=0, use_graph=True):
        L = _lib.load()
        self.ctx = ctx
        cfg = _lib.ExecConfig(int(tile_width), int(pairs_per_thread), int(core_block_sites),
                              int(flank_sites), int(max_window_sites), int(max_tasks),
                              int(max_pool_bytes), int(max_ctas), 1 if use_graph else 0)
        self.config = {"tile_width": int(tile_width), "pairs_per_thread": int(pairs_per_thread),
                       "core_block_sites": int(core_block_sites),
                       "flank_sites": int(flank_sites), "use_graph": bool(use_graph)}
        h = ctypes.c_void_p()
        check(L.gsmc_exec_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        g = ctypes.c_int()
        pb = ctypes.c_uint64()
        rows = ctypes.c_int64()
        mt = ctypes.c_int64()
        check(L.gsmc_exec_info(h, ctypes.byref(g), ctypes.byref(pb), ctypes.byref(rows),
                               ctypes.byref(mt)))
        self.grid, self.pool_bytes = int(g.value), int(pb.value)
        self.slot_rows, self.max_tasks = int(rows.value), int(mt.value)

    @property
    def handle(self):
        return self._h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.gsmc_exec_destroy(h)
        self._h = None

    __del__ = close

    def run(self, layout, pair_base, out_base, stream_handle):
        """Enqueue the jobs of ``layout`` whose pairs/outputs live at the given
        device addresses on ``stream_handle`` (a cudaStream_t as int)."""
        arr = layout.c_jobs(pair_base, out_base)
        check(_lib.load().gsmc_exec_run(self._h, arr, len(layout.jobs), stream_handle))

    def timing(self, enable):
        check(_lib.load().gsmc_exec_timing(self._h, 1 if enable else 0))

    def timing_read(self):
        """(kernel ms, launches, pair-sites) since the last read."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        ps = ctypes.c_double()
        check(_lib.load().gsmc_exec_timing_read(self._h, ctypes.byref(ms), ctypes.byref(n),
                                                ctypes.byref(ps)))
        return float(ms.value), int(n.value), float(ps.value)


class DeviceBatch:
    """Device (and pinned host) buffers of one batch of jobs."""

    def __init__(self, layout, device):
        import torch
        self.layout = layout
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.h_pairs = torch.empty(max(layout.pair_ints, 1), dtype=torch.int32, pin_memory=True)
        layout.pack_pairs(self.h_pairs.numpy())
        self.d_pairs = None
        self.d_out = None
        self.h_out = None
        self.done = None

    def allocate(self, stream):
        """Device buffers, allocated on the stream that will use them."""
        import torch
        with torch.cuda.stream(stream):
            self.d_pairs = torch.empty(max(self.layout.pair_ints, 1), dtype=torch.int32,
                                       device=self.device)
            self.d_out = torch.empty(max(self.layout.out_floats, 1), dtype=torch.float32,
                                     device=self.device)

    def launch(self, executor, stream):
        """Upload pairs, run the jobs, copy every output back to pinned host
        memory, all on ``stream``; returns the completion event."""
        import torch
        if self.d_out is None:
            self.allocate(stream)
        with torch.cuda.stream(stream):
            self.d_pairs.copy_(self.h_pairs, non_blocking=True)
            executor.run(self.layout, self.d_pairs.data_ptr(), self.d_out.data_ptr(),
                         stream.cuda_stream)
            self.h_out = torch.empty(self.d_out.numel(), dtype=torch.float32, pin_memory=True)
            self.h_out.copy_(self.d_out, non_blocking=True)
            self.done = torch.cuda.Event()
            self.done.record(stream)
        return self.done

    def results(self):
        """Per-job result dicts (views into the pinned host buffer); waits."""
        self.done.synchronize()
        return self.layout.results(self.h_out.numpy())


def run_jobs(ctx, jobs, executor=None, stream=None, **config):
    """Run ``jobs`` on ``ctx`` in one persistent launch and return one result
    dict per job (``mean`` and, as selected, ``lower``/``upper``,
    ``posterior_alpha``/``posterior_beta``; each ``[rows, n_pairs]`` float32)."""
    import torch
    jobs = [j if isinstance(j, Job) else Job(**j) for j in jobs]
    for j in jobs:
        validate(j, ctx.n_haps, ctx.n_sites)
    own = executor is None
    if own:
        config.setdefault("max_tasks", max(1 << 10, _count_tasks(jobs, config)))
        if int(config.get("core_block_sites", 0)) <= 0:
            config.setdefault("max_window_sites", max([j.rows for j in jobs] + [1]))
        executor = Executor(ctx, **config)
    try:
        device = torch.device("cuda", ctx.device_id)
        stream = stream or torch.cuda.current_stream(device)
        b = DeviceBatch(Layout(jobs), device)
        b.launch(executor, stream)
        return b.results()
    finally:
        if own:
            executor.close()


def _count_tasks(jobs, config):
    """Upper bound of the tasks an executor with ``config`` makes of ``jobs``."""
    core = int(config.get("core_block_sites", 0))
    tile = int(config.get("tile_width", 32)) * int(config.get("pairs_per_thread", 1))
    n = 0
    for j in jobs:
        chunks = 1 if core <= 0 else -(-max(j.rows, 1) // core)
        n += chunks * -(-j.n_pairs // tile)
    return n
