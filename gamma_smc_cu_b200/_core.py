"""Python face of the CUDA library with the reference's ``_core`` names.

``FlowContext``, ``cuda_mem_info``, ``set_device``, ``get_device``,
``get_device_count``, ``bitpack`` and ``unpack`` keep the signatures, defaults,
result dictionaries and error types of the reference's pybind11 module
(src/bindings.cpp:3630-3652, 3687-3730) and call ``lib/libgsmc_b200.so``
through its C ABI (include/gsmc_b200.h).  ``infer.py`` looks these names up
on this module at call time, so tests can monkeypatch them.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

from . import _lib
from ._lib import GSMC_CI, GSMC_POSTERIOR, check, ptr

DEFAULT_FLOW_FIELD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                  "default_flow_field.txt")


def cuda_mem_info():
    """(free_bytes, total_bytes) of the current CUDA device."""
    L = _lib.load()
    f = ctypes.c_uint64()
    t = ctypes.c_uint64()
    check(L.gsmc_mem_info(ctypes.byref(f), ctypes.byref(t)))
    return int(f.value), int(t.value)


def get_device_count():
    n = ctypes.c_int()
    check(_lib.load().gsmc_get_device_count(ctypes.byref(n)))
    return int(n.value)


def set_device(device_id):
    check(_lib.load().gsmc_set_device(int(device_id)))


def get_device():
    d = ctypes.c_int()
    check(_lib.load().gsmc_get_device(ctypes.byref(d)))
    return int(d.value)


def bitpack(G):
    """Pack haplotypes into uint64 words, [n, ceil(S/64)] (bit b of word w = site 64w+b)."""
    G = np.ascontiguousarray(G, dtype=np.uint8)
    if G.ndim != 2:
        raise RuntimeError("G must be 2D (n x S)")
    n, S = G.shape
    out = np.zeros((n, (S + 63) // 64), np.uint64)
    check(_lib.load().gsmc_bitpack(ptr(G, _lib.c_u8p), n, S, ptr(out, _lib.c_u64p)))
    return out


def unpack(packed, n, S):
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    out = np.zeros((int(n), int(S)), np.uint8)
    check(_lib.load().gsmc_unpack(ptr(packed, _lib.c_u64p), int(n), int(S),
                                  ptr(out, _lib.c_u8p)))
    return out


def diploid_het_counts(G):
    """int64 [n_haps // 2]: sites where haplotypes 2k and 2k+1 differ, counted
    on the GPU (bit-packed XOR + popcount); the calibration sums of
    infer.py:44-99."""
    G = np.ascontiguousarray(G, dtype=np.uint8)
    if G.ndim != 2:
        raise ValueError("G must be 2D (n_haplotypes x n_sites)")
    n, S = G.shape
    out = np.zeros(n // 2, np.int64)
    check(_lib.load().gsmc_diploid_het_counts(ptr(G, _lib.c_u8p), n, S, ptr(out, _lib.c_i64p)))
    return out


def gamma_smc_flow_fb(G, positions, pairs, Ne=10000.0, mu=1.25e-8, rho=1e-8,
                      flow_field_path=DEFAULT_FLOW_FIELD, mean_only=False):
    """Uncached flow-field forward-backward (the reference's module-level
    ``gamma_smc_flow_fb``, src/bindings.cpp:2159-2300): every gap integrated on
    the flow field staged in shared memory, raw (mu, rho).  Dict with ``mean``
    (and ``lower``/``upper`` unless mean_only), [n_sites, n_pairs] float32."""
    G = np.ascontiguousarray(G, dtype=np.uint8)
    positions = np.ascontiguousarray(positions, dtype=np.float64)
    if G.ndim != 2 or positions.ndim != 1 or positions.shape[0] != G.shape[1]:
        raise ValueError("G must be [n_haplotypes, n_sites] and positions [n_sites]")
    n, S = G.shape
    pi, pj = _split_pairs(pairs)
    P = len(pi)
    out = {"mean": np.empty((S, P), np.float32)}
    if not mean_only:
        out["lower"] = np.empty((S, P), np.float32)
        out["upper"] = np.empty((S, P), np.float32)
    check(_lib.load().gsmc_flow_fb(
        ptr(G, _lib.c_u8p), n, S, ptr(positions, _lib.c_f64p), ptr(pi, _lib.c_i32p),
        ptr(pj, _lib.c_i32p), P, float(Ne), float(mu), float(rho),
        os.fsencode(str(flow_field_path)), 0 if mean_only else GSMC_CI,
        ptr(out["mean"], _lib.c_f32p), ptr(out.get("lower"), _lib.c_f32p),
        ptr(out.get("upper"), _lib.c_f32p)))
    return out


_RESULT_MEMORY = os.environ.get("GSMC_RESULT_MEMORY", "pageable")


def set_result_memory(kind):
    """Where the host result arrays of this module's calls live (no reference
    counterpart).  "pageable" (default): fresh numpy arrays, filled through
    the library's pinned staging ring by host threads.  "pinned": arrays in
    page-locked buffers that the device-to-host DMA writes directly; a buffer
    returns to a cache when its last array is dropped and is reused by later
    calls it fits, so repeated large calls skip both the staging copy and the
    first-touch page faults.  Allocating page-locked memory the first time is
    slow (seconds per 100 GB), so "pinned" pays off from the second call of a
    size on.  Returns the previous setting."""
    global _RESULT_MEMORY
    if kind not in ("pageable", "pinned"):
        raise ValueError("result memory must be 'pageable' or 'pinned'")
    prev, _RESULT_MEMORY = _RESULT_MEMORY, kind
    return prev


def _free_host(ptr):
    if _lib._lib is not None:
        _lib._lib.gsmc_host_free(ctypes.c_void_p(ptr))


class _HostBlock:
    """A page-locked buffer from the library's cache; numpy views keep it
    alive and it returns to the cache when the last one goes."""

    def __init__(self, nbytes):
        p = ctypes.c_void_p()
        check(_lib.load().gsmc_host_alloc(int(nbytes), ctypes.byref(p)))
        self.__array_interface__ = {"shape": (int(nbytes) // 4,), "typestr": "<f4",
                                    "data": (p.value, False), "version": 3}
        weakref.finalize(self, _free_host, p.value)


# Pageable results at least this large are mapped with transparent huge pages
# requested (GSMC_HUGEPAGES=0 turns that off).
_HUGE_MIN_BYTES = 64 << 20
_HUGEPAGES = os.environ.get("GSMC_HUGEPAGES", "1") != "0"


def _empty_huge(shape, n):
    """A fresh float32 array in an anonymous mapping advised MADV_HUGEPAGE.

    The host copier's threads fault in every page of a fresh result as they
    fill it; at 4 KB a page that is one fault per 4 KB (23 million for a
    93 GB result), at 2 MB one per 2 MB.  Where the kernel does not offer
    transparent huge pages the advice is ignored and the array behaves like
    np.empty's.  The mapping is unmapped when the last view is dropped."""
    import mmap
    # a whole number of 2 MB pages: the kernel places such mappings on a 2 MB
    # boundary, so every page of the array can be a huge one
    size = -(-4 * n // (2 << 20)) * (2 << 20)
    try:
        m = mmap.mmap(-1, size, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
    except (OSError, ValueError):   # no mapping: np.empty's memory (or its MemoryError)
        return np.empty(shape, np.float32)
    try:
        m.madvise(mmap.MADV_HUGEPAGE)
    except (AttributeError, OSError, ValueError):
        pass
    return np.frombuffer(m, np.float32, count=n).reshape(shape)


def _empty(shape):
    """float32 result array of ``shape`` in the memory set_result_memory chose."""
    n = int(np.prod(shape))
    if _RESULT_MEMORY == "pinned" and n > 0:
        return np.asarray(_HostBlock(4 * n))[:n].reshape(shape)
    if _HUGEPAGES and 4 * n >= _HUGE_MIN_BYTES and hasattr(os, "sysconf"):
        return _empty_huge(shape, n)
    return np.empty(shape, np.float32)


def free_cached_tables():
    """Free the scan-table sets no live context holds (the most recently
    released set of each device otherwise stays resident for the next context
    with the same parameters); no reference counterpart."""
    check(_lib.load().gsmc_free_cached_tables())


def _split_pairs(pairs):
    """List of (i, j) (or an (P, 2) array) -> two contiguous int32 arrays."""
    if isinstance(pairs, np.ndarray):
        arr = np.asarray(pairs)
        if arr.size == 0:
            arr = arr.reshape(0, 2)
        if arr.ndim != 2 or arr.shape[1] != 2:
            raise TypeError("pairs must be a sequence of (i, j) pairs")
        return (np.ascontiguousarray(arr[:, 0], np.int32),
                np.ascontiguousarray(arr[:, 1], np.int32))
    pi = np.fromiter((int(p[0]) for p in pairs), dtype=np.int32)
    pj = np.fromiter((int(p[1]) for p in pairs), dtype=np.int32)
    return pi, pj


class FlowContext:
    """Resident genotypes, positions and flow-field tables on the current GPU.

    Same constructor and methods as the reference's ``_core.FlowContext``
    (src/bindings.cpp:2445-3346); the flow field defaults to the bundled
    ``data/default_flow_field.txt``.
    """

    def __init__(self, G, positions, Ne=10000.0, mu=1.25e-8, rho=1e-8,
                 flow_field_path=DEFAULT_FLOW_FIELD, cache_steps=0, table_build="host_fp32"):
        """``table_build`` (no reference counterpart): "host_fp32" builds the
        scan tables on the host exactly as the reference does (bit-identical
        results); "gpu_fp64" builds them on the GPU in float64."""
        L = _lib.load()
        if table_build not in ("host_fp32", "gpu_fp64"):
            raise ValueError("table_build must be 'host_fp32' or 'gpu_fp64'")
        G = np.ascontiguousarray(G, dtype=np.uint8)
        positions = np.ascontiguousarray(positions, dtype=np.float64)
        if G.ndim != 2:
            raise ValueError("G must be 2D (n_haplotypes x n_sites)")
        n, S = G.shape
        if positions.ndim != 1 or positions.shape[0] != S:
            raise ValueError("positions length must match the number of sites in G")
        h = ctypes.c_void_p()
        flags = _lib.GSMC_TABLES_GPU_F64 if table_build == "gpu_fp64" else 0
        check(L.gsmc_ctx_create_ex(ptr(G, _lib.c_u8p), n, S, ptr(positions, _lib.c_f64p),
                                   float(Ne), float(mu), float(rho),
                                   os.fsencode(str(flow_field_path)), int(cache_steps), flags,
                                   ctypes.byref(h)))
        self._h = h
        self._n = n
        self._S = S
        d = ctypes.c_int()
        check(L.gsmc_ctx_info(h, ctypes.byref(d), None, None))
        self._device = int(d.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.gsmc_ctx_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    @property
    def handle(self):
        return self._h

    @property
    def device_id(self):
        return self._device

    @property
    def n_haps(self):
        return self._n

    @property
    def n_sites(self):
        return self._S

    def _outputs(self, rows, P, ci, posterior):
        out = {"mean": _empty((rows, P))}
        if ci:
            out["lower"] = _empty((rows, P))
            out["upper"] = _empty((rows, P))
        if posterior:
            out["posterior_alpha"] = _empty((rows, P))
            out["posterior_beta"] = _empty((rows, P))
        return out

    @staticmethod
    def _out_ptrs(out):
        return [ptr(out.get(k), _lib.c_f32p) for k in
                ("mean", "lower", "upper", "posterior_alpha", "posterior_beta")]

    def run_fb(self, pairs, mean_only=True, return_posterior=False):
        """Full-sequence forward-backward; dict of [n_sites, n_pairs] float32."""
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        if P == 0:
            return self._outputs(self._S, 0, False, return_posterior)
        ci = not mean_only
        out = self._outputs(self._S, P, ci, return_posterior)
        flags = (GSMC_CI if ci else 0) | (GSMC_POSTERIOR if return_posterior else 0)
        check(_lib.load().gsmc_run_fb(self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p), P,
                                      flags, *self._out_ptrs(out)))
        return out

    def run_fb_window(self, pairs, site_begin, site_end, mean_only=True,
                      return_posterior=False):
        """Forward-backward over sites [site_begin, site_end) only, decoded as
        one padded window of the reference's block kernels (a window that does
        not start at site 0 enters its first site by 1 bp); dict of
        [site_end - site_begin, n_pairs] float32.  One call per query."""
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        rows = int(site_end) - int(site_begin)
        if rows < 0 or site_begin < 0 or site_end > self._S:
            raise ValueError(f"site window [{site_begin}, {site_end}) is out of range for "
                             f"{self._S} sites")
        ci = not mean_only
        out = self._outputs(rows, P, ci, return_posterior)
        if P == 0 or rows == 0:
            return out
        flags = (GSMC_CI if ci else 0) | (GSMC_POSTERIOR if return_posterior else 0)
        check(_lib.load().gsmc_run_fb_window(self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p),
                                             P, int(site_begin), int(site_end), flags,
                                             *self._out_ptrs(out)))
        return out

    def run_fwd(self, pairs, mean_only=True):
        """Forward-only (filtered) posterior, the reference's ``run_fwd``:
        dict with ``mean`` (and ``lower``/``upper`` unless mean_only) of shape
        [n_sites, n_pairs] float32."""
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        if P == 0:
            return {"mean": np.empty((self._S, 0), np.float32)}
        out = {"mean": np.empty((self._S, P), np.float32)}
        if not mean_only:
            out["lower"] = np.empty((self._S, P), np.float32)
            out["upper"] = np.empty((self._S, P), np.float32)
        check(_lib.load().gsmc_run_fwd(self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p), P,
                                       0 if mean_only else GSMC_CI,
                                       ptr(out["mean"], _lib.c_f32p),
                                       ptr(out.get("lower"), _lib.c_f32p),
                                       ptr(out.get("upper"), _lib.c_f32p)))
        return out

    def run_fb_blockwise_stream(self, pairs, sink, core_block_sites=8192, flank_sites=2048,
                                pair_batch_size=-1, mean_only=True, return_posterior=False,
                                max_chunk_bytes=1 << 30):
        """Blockwise forward-backward streamed to ``sink`` instead of returned:
        ``sink(site_begin, site_end, pair_begin, pair_end, outputs)`` is called
        once per (window, pair chunk) with a dict of [site_end - site_begin,
        pair_end - pair_begin] float32 views (``mean`` and, as selected,
        ``lower``/``upper``, ``posterior_alpha``/``posterior_beta``) into pinned
        staging that is reused after the call -- copy what must outlive it.
        A sink returning True stops the stream (ValueError).  For results
        larger than host memory; values equal run_fb_blockwise's."""
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        keys = ["mean"] + (["lower", "upper"] if not mean_only else []) + \
            (["posterior_alpha", "posterior_beta"] if return_posterior else [])
        flags = (GSMC_CI if not mean_only else 0) | (GSMC_POSTERIOR if return_posterior else 0)
        index = {"mean": 0, "lower": 1, "upper": 2, "posterior_alpha": 3, "posterior_beta": 4}
        errors = []

        def trampoline(user, s0, s1, p0, p1, outs, ld):
            try:
                rows, n = s1 - s0, p1 - p0
                views = {k: np.ctypeslib.as_array(outs[index[k]], shape=(rows * ld,))[:rows * ld]
                         .reshape(rows, ld)[:, :n] for k in keys}
                return 1 if sink(int(s0), int(s1), int(p0), int(p1), views) else 0
            except BaseException as e:  # reported after the stream stops
                errors.append(e)
                return 1

        cb = _lib.SINK_FN(trampoline)
        rc = _lib.load().gsmc_run_fb_blockwise_stream(
            self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p), P, int(core_block_sites),
            int(flank_sites), int(pair_batch_size), flags, cb, None, int(max_chunk_bytes))
        if errors:
            raise errors[0]
        check(rc)

    def run_fb_summary(self, pairs, core_block_sites=0, flank_sites=2048, pair_batch_size=-1):
        """Per-site mean / min / max over the pairs of the posterior mean, with
        no [n_sites, n_pairs] output (reference ``run_fb_summary``; the
        reference's site_min/site_max are left unwritten there, here they are
        the extremes over the pairs).  ``core_block_sites > 0`` decodes
        blockwise.  Returns site_mean, site_min, site_max ([n_sites] float32)
        and n_pairs."""
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        if P == 0:
            return {"site_mean": np.zeros(0, np.float32)}
        out = {k: np.empty(self._S, np.float32) for k in ("site_mean", "site_min", "site_max")}
        check(_lib.load().gsmc_run_fb_summary(
            self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p), P, int(core_block_sites),
            int(flank_sites), int(pair_batch_size), ptr(out["site_mean"], _lib.c_f32p),
            ptr(out["site_min"], _lib.c_f32p), ptr(out["site_max"], _lib.c_f32p)))
        out["n_pairs"] = P
        return out

    def run_fb_blockwise(self, pairs, core_block_sites=8192, flank_sites=2048,
                         pair_batch_size=256, max_streams=1, mean_only=True,
                         return_posterior=False):
        """Blockwise forward-backward over flanked windows; adds ``blocks``."""
        L = _lib.load()
        # argument checks precede everything, as in src/bindings.cpp:3000-3016
        if core_block_sites <= 0:
            raise ValueError("core_block_sites must be positive.")
        if flank_sites < 0:
            raise ValueError("flank_sites must be non-negative.")
        if pair_batch_size == 0 or pair_batch_size < -1:
            raise ValueError("pair_batch_size must be positive or -1 for auto.")
        if max_streams <= 0:
            raise ValueError("max_streams must be positive.")
        if return_posterior and max_streams > 1:
            raise ValueError(
                "return_posterior=True is currently only supported with max_streams=1. "
                "Run blockwise posterior decoding in single-stream mode.")
        pi, pj = _split_pairs(pairs)
        P = len(pi)
        nb = ctypes.c_int64()
        check(L.gsmc_block_count(self._S, int(core_block_sites), ctypes.byref(nb)))
        blocks = np.zeros((nb.value, 4), np.int32)
        if P == 0:
            out = self._outputs(self._S, 0, False, return_posterior)
        elif nb.value == 0:
            out = self._outputs(0, P, False, return_posterior)
        else:
            out = self._outputs(self._S, P, not mean_only, return_posterior)
        flags = (GSMC_CI if not mean_only else 0) | (GSMC_POSTERIOR if return_posterior else 0)
        if P == 0 or nb.value == 0:
            flags = 0
        check(L.gsmc_run_fb_blockwise(
            self._h, ptr(pi, _lib.c_i32p), ptr(pj, _lib.c_i32p), P, int(core_block_sites),
            int(flank_sites), int(pair_batch_size), int(max_streams), flags,
            ptr(blocks, _lib.c_i32p), *self._out_ptrs(out)))
        result = {"blocks": blocks}
        result.update(out)
        return result

    def release_scratch(self):
        """Free the device scratch the context keeps between calls (forward-
        state slots, stages); genotypes and tables stay.  No reference
        counterpart."""
        check(_lib.load().gsmc_ctx_release_scratch(self._h))

    def scan_shape(self):
        """(threads per task, pairs per thread) of the context's latest scan
        launch; no reference counterpart."""
        w, k = ctypes.c_int(), ctypes.c_int()
        check(_lib.load().gsmc_ctx_scan_shape(self._h, ctypes.byref(w), ctypes.byref(k)))
        return int(w.value), int(k.value)

    def spec_stats(self):
        """(launches cut into exact speculative site chunks, (window, pair)s
        decoded again whole after a failed boundary check) of this context so
        far; no reference counterpart."""
        a, r = ctypes.c_int64(), ctypes.c_int64()
        check(_lib.load().gsmc_ctx_spec_stats(self._h, ctypes.byref(a), ctypes.byref(r)))
        return int(a.value), int(r.value)

    def tables_info(self):
        """{"build_seconds": build + upload of this context's scan tables (0.0
        when it reused a resident set), "reused": bool}; no reference
        counterpart."""
        secs, reused = ctypes.c_double(), ctypes.c_int()
        check(_lib.load().gsmc_ctx_tables_info(self._h, ctypes.byref(secs), ctypes.byref(reused)))
        return {"build_seconds": float(secs.value), "reused": bool(reused.value)}

    def table_layer(self, table, layer):
        """Debug: (m_grid, c_grid) [51, 50] of scan table 0..4 at a layer."""
        buf = np.empty(2 * 2550, np.float32)
        check(_lib.load().gsmc_ctx_table_layer(self._h, int(table), int(layer),
                                               ptr(buf, _lib.c_f32p)))
        return buf[:2550].reshape(51, 50), buf[2550:].reshape(51, 50)
