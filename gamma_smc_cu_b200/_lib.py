"""ctypes binding of the in-tree CUDA library ``lib/libgsmc_b200.so``.

The library is the product: there is no CPU fallback.  If it has not been
built, every entry point raises at first use (``python -m
gamma_smc_cu_b200.build`` builds it; nvcc cross-compiles without a GPU).
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GSMC_LIB_PATH") or os.path.join(HERE, "lib", "libgsmc_b200.so")

GSMC_OK = 0
GSMC_E_INVALID = -1
GSMC_E_CUDA = -2
GSMC_E_IO = -3
GSMC_E_NOMEM = -4
GSMC_E_TIMEOUT = -5

GSMC_CI = 1
GSMC_POSTERIOR = 2

GSMC_TABLES_GPU_F64 = 1

c_i64 = ctypes.c_int64
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_vp = ctypes.c_void_p
c_int = ctypes.c_int
c_intp = ctypes.POINTER(ctypes.c_int)

class ExecConfig(ctypes.Structure):
    """gsmc_exec_config of include/gsmc_b200.h."""
    _fields_ = [
        ("tile_width", ctypes.c_int32),
        ("pairs_per_thread", ctypes.c_int32),
        ("core_block_sites", ctypes.c_int64),
        ("flank_sites", ctypes.c_int64),
        ("max_window_sites", ctypes.c_int64),
        ("max_tasks", ctypes.c_int64),
        ("max_pool_bytes", ctypes.c_uint64),
        ("max_ctas", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
    ]


class Job(ctypes.Structure):
    """gsmc_job of include/gsmc_b200.h (device pointers as integers)."""
    _fields_ = [
        ("pair_i", ctypes.c_void_p),
        ("pair_j", ctypes.c_void_p),
        ("n_pairs", ctypes.c_int64),
        ("site_begin", ctypes.c_int64),
        ("site_end", ctypes.c_int64),
        ("flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("out", ctypes.c_void_p * 5),
        ("ld_out", ctypes.c_int64),
        ("out_col0", ctypes.c_int64),
    ]


# gsmc_sink_fn: (user, site_begin, site_end, pair_begin, pair_end, outputs[5], ld) -> int
SINK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                           ctypes.c_int64, ctypes.c_int64,
                           ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.c_int64)

# name -> (restype, argtypes); mirrors include/gsmc_b200.h
SIGNATURES = {
    "gsmc_last_error": (ctypes.c_char_p, []),
    "gsmc_version": (ctypes.c_char_p, []),
    "gsmc_mem_info": (c_int, [c_u64p, c_u64p]),
    "gsmc_get_device_count": (c_int, [c_intp]),
    "gsmc_set_device": (c_int, [c_int]),
    "gsmc_get_device": (c_int, [c_intp]),
    "gsmc_ctx_create": (c_int, [c_u8p, c_i64, c_i64, c_f64p, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_char_p, c_int, ctypes.POINTER(c_vp)]),
    "gsmc_ctx_create_ex": (c_int, [c_u8p, c_i64, c_i64, c_f64p, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_char_p, c_int, c_int,
                                   ctypes.POINTER(c_vp)]),
    "gsmc_ctx_destroy": (c_int, [c_vp]),
    "gsmc_ctx_info": (c_int, [c_vp, c_intp, c_i64p, c_i64p]),
    "gsmc_run_fb": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_int, c_f32p, c_f32p, c_f32p,
                            c_f32p, c_f32p]),
    "gsmc_block_count": (c_int, [c_i64, c_i64, c_i64p]),
    "gsmc_run_fb_blockwise": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_i64, c_i64, c_i64, c_int,
                                      c_int, c_i32p, c_f32p, c_f32p, c_f32p, c_f32p, c_f32p]),
    "gsmc_run_fb_blockwise_device": (c_int, [c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_int, c_vp,
                                             c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_vp]),
    "gsmc_run_fb_blockwise_device_noalloc": (c_int, [c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_int,
                                                     c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_i64,
                                                     c_vp]),
    "gsmc_run_fb_window": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_i64, c_i64, c_int, c_f32p,
                                   c_f32p, c_f32p, c_f32p, c_f32p]),
    "gsmc_exec_create": (c_int, [c_vp, ctypes.POINTER(ExecConfig), ctypes.POINTER(c_vp)]),
    "gsmc_exec_destroy": (c_int, [c_vp]),
    "gsmc_exec_info": (c_int, [c_vp, c_intp, c_u64p, c_i64p, c_i64p]),
    "gsmc_exec_run": (c_int, [c_vp, ctypes.POINTER(Job), c_i64, c_vp]),
    "gsmc_exec_run_checked": (c_int, [c_vp, ctypes.POINTER(Job), c_i64, c_vp, c_vp]),
    "gsmc_exec_timing": (c_int, [c_vp, c_int]),
    "gsmc_exec_timing_read": (c_int, [c_vp, ctypes.POINTER(ctypes.c_double), c_i64p,
                                      ctypes.POINTER(ctypes.c_double)]),
    "gsmc_copy_to_host": (c_int, [c_i64, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp), c_u64p,
                                  c_vp]),
    "gsmc_run_fb_summary": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_i64, c_i64, c_i64, c_f32p,
                                    c_f32p, c_f32p]),
    "gsmc_run_fwd": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_int, c_f32p, c_f32p, c_f32p]),
    "gsmc_diploid_het_counts": (c_int, [c_u8p, c_i64, c_i64, c_i64p]),
    "gsmc_generate_flow_field": (c_int, [c_f64p, c_f64p, c_int, c_int, c_int, c_int, c_f64p,
                                         c_f64p, c_f64p, ctypes.c_double, c_f64p, c_f64p]),
    "gsmc_flow_fb": (c_int, [c_u8p, c_i64, c_i64, c_f64p, c_i32p, c_i32p, c_i64, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, ctypes.c_char_p, c_int, c_f32p,
                             c_f32p, c_f32p]),
    "gsmc_run_fb_blockwise_stream": (c_int, [c_vp, c_i32p, c_i32p, c_i64, c_i64, c_i64, c_i64,
                                             c_int, SINK_FN, c_vp, ctypes.c_uint64]),
    "gsmc_ctx_spec_stats": (c_int, [c_vp, c_i64p, c_i64p]),
    "gsmc_ctx_scan_shape": (c_int, [c_vp, c_i32p, c_i32p]),
    "gsmc_flow_fb_stats": (c_int, [c_i32p, c_i64p]),
    "gsmc_ctx_release_scratch": (c_int, [c_vp]),
    "gsmc_ctx_scratch_bytes": (c_int, [c_vp, c_u64p]),
    "gsmc_ctx_timing": (c_int, [c_vp, c_int]),
    "gsmc_ctx_timing_read": (c_int, [c_vp, ctypes.POINTER(ctypes.c_double), c_i64p,
                                     ctypes.POINTER(ctypes.c_double)]),
    "gsmc_set_copy_wait_polls": (c_int, [c_i64, c_i64p]),
    "gsmc_ctx_tables_info": (c_int, [c_vp, ctypes.POINTER(ctypes.c_double), c_intp]),
    "gsmc_free_cached_tables": (c_int, []),
    "gsmc_host_alloc": (c_int, [ctypes.c_uint64, ctypes.POINTER(c_vp)]),
    "gsmc_host_free": (c_int, [c_vp]),
    "gsmc_host_cache_limit": (c_int, [ctypes.c_uint64]),
    "gsmc_bitpack": (c_int, [c_u8p, c_i64, c_i64, c_u64p]),
    "gsmc_unpack": (c_int, [c_u64p, c_i64, c_i64, c_u8p]),
    "gsmc_ctx_table_layer": (c_int, [c_vp, c_int, c_int, c_f32p]),
}

_lib = None
_lock = threading.Lock()


class GsmcError(RuntimeError):
    pass


def load():
    """Load the CUDA library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"gamma_smc_cu_b200: CUDA library not built ({LIB_PATH}); "
                    "run `python -m gamma_smc_cu_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error():
    return load().gsmc_last_error().decode(errors="replace")


def check(rc):
    """Map a status code to the exception the reference raised for it."""
    if rc == GSMC_OK:
        return
    msg = last_error()
    if rc == GSMC_E_INVALID:
        raise ValueError(msg)
    if rc == GSMC_E_NOMEM:
        raise MemoryError(msg)
    raise GsmcError(msg)


def ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)
