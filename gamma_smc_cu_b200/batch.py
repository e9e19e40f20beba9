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
    def layout_floats(self):
        """Floats the job's outputs take in a batch buffer (each output
        region padded to the 64-float alignment of Layout)."""
        return -(-(self.rows * self.n_pairs) // _ALIGN) * _ALIGN * self.n_outputs

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


# numpy image of gsmc_job (include/gsmc_b200.h), so a batch's descriptors are
# built with array operations instead of one ctypes field at a time
JOB_DTYPE = np.dtype([("pair_i", "<u8"), ("pair_j", "<u8"), ("n_pairs", "<i8"),
                      ("site_begin", "<i8"), ("site_end", "<i8"), ("flags", "<i4"),
                      ("reserved", "<i4"), ("out", "<u8", (5,)), ("ld_out", "<i8"),
                      ("out_col0", "<i8")])
_ALIGN = 64  # floats: every output region starts on a 256-byte boundary


class Layout:
    """Where each job's pairs and outputs sit in one flat batch buffer.

    Pairs: int32 ``[pi of job 0 | pj of job 0 | pi of job 1 | ...]``.
    Outputs: float32, per job its selected outputs in OUTPUT_KEYS order, each
    ``[rows, n_pairs]`` row-major, 64-float aligned.
    """

    def __init__(self, jobs):
        self.jobs = list(jobs)
        J = len(self.jobs)
        n = np.fromiter((j.n_pairs for j in self.jobs), np.int64, J)
        rows = np.fromiter((j.rows for j in self.jobs), np.int64, J)
        sel = np.array([_selected(j.mean_only, j.return_posterior) for j in self.jobs],
                       dtype=bool).reshape(J, 5)
        self.n_pairs, self.rows, self.sel = n, rows, sel
        self.pair_off = np.concatenate([[0], np.cumsum(2 * n)[:-1]]) if J else n
        size = -(-(rows * n) // _ALIGN) * _ALIGN
        sizes = np.where(sel, size[:, None], 0).ravel()
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]) if J else sizes
        self.out_off = np.where(sel.ravel(), offs, -1).reshape(J, 5)
        self.pair_ints = int(2 * n.sum())
        self.out_floats = int(sizes.sum())
        self.flags = np.fromiter((j.flags for j in self.jobs), np.int32, J)

    def pack_pairs(self, dst):
        """Write every job's pairs into the int32 array ``dst``."""
        if self.jobs:
            parts = [p for j in self.jobs for p in (j.pairs[:, 0], j.pairs[:, 1])]
            dst[:self.pair_ints] = np.concatenate(parts)

    def job_array(self, pair_base, out_base):
        """gsmc_job records (JOB_DTYPE) for device buffers at the given addresses."""
        J = len(self.jobs)
        a = np.zeros(J, JOB_DTYPE)
        a["pair_i"] = pair_base + 4 * self.pair_off
        a["pair_j"] = pair_base + 4 * (self.pair_off + self.n_pairs)
        a["n_pairs"] = self.n_pairs
        a["site_begin"] = [j.site_begin for j in self.jobs]
        a["site_end"] = [j.site_end for j in self.jobs]
        a["flags"] = self.flags
        a["out"] = np.where(self.out_off >= 0, out_base + 4 * self.out_off, 0).astype(np.uint64)
        a["ld_out"] = self.n_pairs
        return a

    def c_jobs(self, pair_base, out_base):
        """ctypes view (gsmc_job array) of job_array; keeps the array alive."""
        a = self.job_array(pair_base, out_base)
        arr = (_lib.Job * len(self.jobs)).from_buffer(a)
        arr._keep = a
        return arr

    def results(self, host):
        """Per-job result dicts of views into the float32 host array."""
        res = []
        for k, j in enumerate(self.jobs):
            d = {}
            for i, key in enumerate(OUTPUT_KEYS):
                o = int(self.out_off[k, i])
                if o >= 0:
                    d[key] = host[o:o + j.rows * j.n_pairs].reshape(j.rows, j.n_pairs)
            res.append(d)
        return res

    def regions(self):
        """(job index, output key, float offset, floats) of every output."""
        out = []
        for k, j in enumerate(self.jobs):
            for i, key in enumerate(OUTPUT_KEYS):
                o = int(self.out_off[k, i])
                if o >= 0 and j.rows * j.n_pairs:
                    out.append((k, key, o, j.rows * j.n_pairs))
        return out


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

    def run(self, layout, pair_base, out_base, stream_handle, flags=None):
        """Enqueue the jobs of ``layout`` whose pairs/outputs live at the given
        device addresses on ``stream_handle`` (a cudaStream_t as int).  With
        ``flags`` (device address of len(jobs) int32) the chunked jobs are
        checked: flags[k] becomes 1 where job k's chunks did not join its
        whole-window decode bit for bit."""
        arr = layout.c_jobs(pair_base, out_base)
        if flags is None:
            check(_lib.load().gsmc_exec_run(self._h, arr, len(layout.jobs), stream_handle))
        else:
            check(_lib.load().gsmc_exec_run_checked(self._h, arr, len(layout.jobs),
                                                    stream_handle, flags))

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
    """Device buffers of one batch of jobs, and where its results go.

    ``launch`` uploads the pairs, runs the jobs and -- when ``host`` is given
    (a pinned float32 array of ``layout.out_floats``) -- copies every output
    into it on the same stream.  Without ``host`` the outputs stay on the
    device; ``to_host`` then copies them into fresh (pageable) numpy arrays
    through the library's pinned ring.

    Chunked jobs are checked on the device: a job whose chunks' boundary
    states did not join its whole-window decode bit for bit (rare; the
    burn-in is ``flank_sites``) is decoded again whole through the context
    when its results are collected, so every result equals
    ``FlowContext.run_fb_window`` for the same query exactly.  ``repaired``
    counts such jobs.
    """

    def __init__(self, layout, device):
        import torch
        self.layout = layout
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.h_pairs = torch.empty(max(layout.pair_ints, 1), dtype=torch.int32, pin_memory=True)
        layout.pack_pairs(self.h_pairs.numpy())
        self.h_flags = torch.zeros(max(len(layout.jobs), 1), dtype=torch.int32, pin_memory=True)
        self.d_flags = None
        self.executor = None
        self.repaired = 0
        self.d_pairs = None
        self.d_out = None
        self.h_out = None
        self.done = None
        self.stream = None

    def allocate(self, stream):
        """Device buffers, allocated on the stream that will use them."""
        import torch
        with torch.cuda.stream(stream):
            self.d_pairs = torch.empty(max(self.layout.pair_ints, 1), dtype=torch.int32,
                                       device=self.device)
            self.d_out = torch.empty(max(self.layout.out_floats, 1), dtype=torch.float32,
                                     device=self.device)
            self.d_flags = torch.zeros(max(len(self.layout.jobs), 1), dtype=torch.int32,
                                       device=self.device)

    def launch(self, executor, stream, host=None):
        """Upload pairs, run the jobs, optionally copy the outputs into the
        pinned array ``host``; all on ``stream``.  Returns the completion event."""
        import torch
        if self.d_out is None:
            self.allocate(stream)
        self.stream = stream
        self.executor = executor
        with torch.cuda.stream(stream):
            self.d_pairs.copy_(self.h_pairs, non_blocking=True)
            executor.run(self.layout, self.d_pairs.data_ptr(), self.d_out.data_ptr(),
                         stream.cuda_stream, flags=self.d_flags.data_ptr())
            self.h_flags.copy_(self.d_flags, non_blocking=True)
            if host is not None:
                self.h_out = host
                n = self.layout.out_floats
                if n:
                    torch.from_numpy(host[:n]).copy_(self.d_out[:n], non_blocking=True)
            self.done = torch.cuda.Event()
            self.done.record(stream)
        return self.done

    def results(self, redo=None):
        """Per-job result dicts (views into the pinned host array); waits.
        Jobs that failed the chunk check are decoded again by ``redo`` (see
        _redo) and written into their views."""
        if self.h_out is None:
            raise RuntimeError("the batch was launched without a host array; use to_host()")
        self.done.synchronize()
        res = self.layout.results(self.h_out)
        for k, exact in self._redo(redo):
            for key, v in res[k].items():
                v[...] = exact[key]
        return res

    def _redo(self, redo=None):
        """(job index, whole-window result) of the jobs whose chunks failed the
        device check, decoded again by ``redo(job)`` (default: the context's
        run_fb_window, so the context must not be busy on another thread);
        call once the batch is done."""
        flags = self.h_flags.numpy()[:len(self.layout.jobs)]
        if redo is None:
            ctx = self.executor.ctx
            redo = lambda j: ctx.run_fb_window(j.pairs, j.site_begin, j.site_end,
                                               mean_only=j.mean_only,
                                               return_posterior=j.return_posterior)
        out = [(int(k), redo(self.layout.jobs[int(k)])) for k in np.flatnonzero(flags)]
        self.repaired = len(out)
        return out

    def to_host(self, redo=None):
        """Per-job result dicts of new numpy arrays, copied from the device
        outputs once the batch is done (no pinned staging of the results)."""
        res = [{} for _ in self.layout.jobs]
        regs = self.layout.regions()
        dst, src, nb = [], [], []
        base = self.d_out.data_ptr()
        for k, key, off, n in regs:
            j = self.layout.jobs[k]
            a = np.empty((j.rows, j.n_pairs), np.float32)
            res[k][key] = a
            dst.append(a.ctypes.data)
            src.append(base + 4 * off)
            nb.append(4 * n)
        for k, j in enumerate(self.layout.jobs):   # empty outputs
            for i, key in enumerate(OUTPUT_KEYS):
                if self.layout.out_off[k, i] >= 0 and key not in res[k]:
                    res[k][key] = np.empty((j.rows, j.n_pairs), np.float32)
        m = len(dst)
        check(_lib.load().gsmc_copy_to_host(
            m, (ctypes.c_void_p * max(m, 1))(*dst), (ctypes.c_void_p * max(m, 1))(*src),
            (ctypes.c_uint64 * max(m, 1))(*nb), self.stream.cuda_stream))
        self.done.synchronize()
        for k, exact in self._redo(redo):
            res[k] = {key: exact[key] for key in res[k]}
        return res


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
        return b.to_host()
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
