"""CPU oracle for the Gamma-SMC cached forward/backward path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product
(``gamma_smc_cu_b200``) never does.  It is the checker, never the thing
measured as the product or shipped.

It restates the reference's host logic in numpy and drives the C++ scan
restatement in ``oracle/gsmc_oracle.cpp`` (built into
``oracle/_build/libgsmc_oracle.so`` by ``oracle/Makefile``):

* ``coerce_inputs``          python/gamma_smc_cu/infer.py:20-41
* ``estimate_scaled_params`` python/gamma_smc_cu/infer.py:44-99
* ``filter_segregating``     python/gamma_smc_cu/infer.py:102-126
* block sizing helpers       python/gamma_smc_cu/infer.py:151-214
* ``make_block_windows``     src/bindings.cpp:2517-2534
* ``infer`` / ``infer_blockwise`` result assembly: infer.py:217-296, 299-484 and
  FlowContext.run_fb / run_fb_blockwise, src/bindings.cpp:2897-3345
* ``pair_to_ij`` / ``ij_to_pair`` include/gamma_smc_cu/types.h:56-68

Parity pin: the restated table builder is compared bit for bit with the
reference's own ``src/flow_field.cpp`` compiled into ``oracle/_ref``; the
restated scan is compared with the reference's compiled ``_core`` on a GPU
(see tests).  The flow field is the fixture
``gamma_smc_cu_b200/data/default_flow_field.txt`` (tests/golden/make_flow_field.py).
"""
from __future__ import annotations

import ctypes
import glob
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgsmc_oracle.so")
REF_TABLES_PATH = os.path.join(HERE, "_ref", "libref_tables.so")

FF_MEAN_N = 51
FF_CV_N = 50
FF_GRID = FF_MEAN_N * FF_CV_N
N_TABLES = 12
TABLE_NAMES = (
    "missing_mean", "missing_cv", "mean", "cv",
    "fwd_hom_site_mean", "fwd_hom_site_cv", "fwd_het_site_mean", "fwd_het_site_cv",
    "bwd_hom_site_mean", "bwd_hom_site_cv", "bwd_het_site_mean", "bwd_het_site_cv",
)
DEFAULT_CACHE_STEPS = 1000  # src/bindings.cpp:2569-2572

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_lib = None
_ref_tables_lib = None


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_load_flow_field.argtypes = [ctypes.c_char_p, _f32p, _f32p, _f32p]
        L.oracle_load_flow_field.restype = ctypes.c_int
        L.oracle_build_tables.argtypes = [_f32p, _f32p, _f32p, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_float, _f32p]
        L.oracle_build_tables.restype = None
        L.oracle_bitpack.argtypes = [_u8p, ctypes.c_longlong, ctypes.c_longlong, _u64p]
        L.oracle_bitpack.restype = None
        L.oracle_fb_window.argtypes = [
            _u64p, ctypes.c_longlong, _f64p, ctypes.c_longlong, ctypes.c_longlong,
            ctypes.c_longlong, _i32p, _i32p, ctypes.c_longlong, ctypes.c_float,
            _f32p, ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_int]
        L.oracle_fb_window.restype = ctypes.c_int
        L.oracle_fwd_only.argtypes = [
            _u64p, ctypes.c_longlong, _f64p, ctypes.c_longlong, _i32p, _i32p, ctypes.c_longlong,
            ctypes.c_float, _f32p, _f32p, ctypes.c_int, _f32p, _f32p, _f32p, ctypes.c_int]
        L.oracle_fwd_only.restype = None
        L.oracle_flow_fb.argtypes = [
            _u64p, ctypes.c_longlong, _f64p, ctypes.c_longlong, _i32p, _i32p, ctypes.c_longlong,
            _f32p, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float, _f32p, _f32p, _f32p,
            ctypes.c_int]
        L.oracle_flow_fb.restype = None
        L.oracle_layer_bilinear.argtypes = [_f32p, ctypes.c_float, ctypes.c_float]
        L.oracle_layer_bilinear.restype = ctypes.c_float
        _lib = L
    return _lib


def layer_bilinear(grid, m, c):
    """The scan's bilinear lookup of (m, c) on a [51, 50] float32 grid."""
    g = np.ascontiguousarray(grid, np.float32).reshape(-1)
    return float(lib().oracle_layer_bilinear(_ptr(g, _f32p), float(m), float(c)))


def ref_tables_lib():
    """The reference's compiled table builder, or None when it was not built."""
    global _ref_tables_lib
    if _ref_tables_lib is None and os.path.exists(REF_TABLES_PATH):
        L = ctypes.CDLL(REF_TABLES_PATH)
        L.ref_load_flow_field.argtypes = [ctypes.c_char_p, _f32p, _f32p, _f32p]
        L.ref_load_flow_field.restype = ctypes.c_int
        L.ref_build_tables.argtypes = [_f32p, _f32p, _f32p, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_float, _f32p]
        L.ref_build_tables.restype = None
        _ref_tables_lib = L
    return _ref_tables_lib


def ref_core_path():
    """Path of the reference's compiled ``_core`` module in oracle/_ref, or None."""
    hits = glob.glob(os.path.join(HERE, "_ref", "_core*.so"))
    return hits[0] if hits else None


# ------------------------------------------------------------------ tables --

def load_flow_field(path, use_reference=False):
    u = np.zeros(FF_GRID, np.float32)
    v = np.zeros(FF_GRID, np.float32)
    b = np.zeros(4, np.float32)
    L = ref_tables_lib() if use_reference else lib()
    fn = L.ref_load_flow_field if use_reference else L.oracle_load_flow_field
    rc = fn(os.fsencode(path), _ptr(u, _f32p), _ptr(v, _f32p), _ptr(b, _f32p))
    if rc != 0:
        raise RuntimeError(f"Failed to load flow field from: {path}")
    return u, v, b


def scaled_rates(Ne, mu, rho):
    """scaled_rho, scaled_mu exactly as the reference forms them in FP32:
    FlowContext casts (Ne, mu, rho) to float (src/bindings.cpp:2575) and
    ensure_cache multiplies 4.0f * Ne * rate (src/bindings.cpp:2044-2045)."""
    f = np.float32
    ne = f(Ne)
    return f(f(f(4.0) * ne) * f(rho)), f(f(f(4.0) * ne) * f(mu))


def build_tables(u, v, bounds, n_steps, Ne, mu, rho, use_reference=False):
    """[12, n_steps, 2550] float32 tables, in TABLE_NAMES order."""
    srho, smu = scaled_rates(Ne, mu, rho)
    out = np.empty((N_TABLES, n_steps, FF_GRID), np.float32)
    L = ref_tables_lib() if use_reference else lib()
    fn = L.ref_build_tables if use_reference else L.oracle_build_tables
    fn(_ptr(u, _f32p), _ptr(v, _f32p), _ptr(bounds, _f32p), int(n_steps),
       float(srho), float(smu), _ptr(out, _f32p))
    return out


_TABLE_CACHE = {}


def tables_for(flow_field_path, Ne, mu, rho, n_steps=DEFAULT_CACHE_STEPS):
    key = (os.path.abspath(flow_field_path), float(np.float32(Ne)),
           float(np.float32(mu)), float(np.float32(rho)), int(n_steps))
    if key not in _TABLE_CACHE:
        u, v, b = load_flow_field(flow_field_path)
        _TABLE_CACHE[key] = build_tables(u, v, b, n_steps, Ne, mu, rho)
    return _TABLE_CACHE[key]


# --------------------------------------------------------------- genotypes --

def bitpack(G):
    G = np.ascontiguousarray(G, dtype=np.uint8)
    n, S = G.shape
    packed = np.zeros((n, (S + 63) // 64), np.uint64)
    lib().oracle_bitpack(_ptr(G, _u8p), n, S, _ptr(packed, _u64p))
    return packed


def unpack(packed, n, S):
    bits = np.unpackbits(packed.view(np.uint8).reshape(n, -1), axis=1, bitorder="little")
    return bits[:, :S].astype(np.uint8)


def pair_to_ij(p):
    """include/gamma_smc_cu/types.h:56-62."""
    r = (1.0 + math.sqrt(1.0 + 8.0 * p)) / 2.0
    i = int(r)
    if i * (i - 1) // 2 > p:
        i -= 1
    return i, p - i * (i - 1) // 2


def ij_to_pair(i, j):
    """include/gamma_smc_cu/types.h:65-68."""
    if i < j:
        i, j = j, i
    return i * (i - 1) // 2 + j


def all_pairs(n):
    """Default pair list of infer(): i > j, row-major (infer.py:272-273)."""
    return [(i, j) for i in range(n) for j in range(i)]


# -------------------------------------------------------------- host logic --

def coerce_inputs(G_or_ts, positions):
    if hasattr(G_or_ts, "genotype_matrix"):
        ts = G_or_ts
        G = ts.genotype_matrix().T.astype(np.uint8, copy=False)
        pos = np.array([v.position for v in ts.variants()], dtype=np.float64)
        return G, pos
    if positions is None:
        raise ValueError("positions is required when G_or_ts is a genotype matrix.")
    G = np.ascontiguousarray(G_or_ts, dtype=np.uint8)
    if G.ndim != 2:
        raise ValueError("G_or_ts must be a 2D haplotype matrix or a tree sequence.")
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    if pos.ndim != 1:
        raise ValueError("positions must be a 1D array of site coordinates.")
    if G.shape[1] != pos.shape[0]:
        raise ValueError("positions length must match the number of sites in G_or_ts.")
    return G, pos


def diploid_het_counts(G):
    """int64 [n // 2]: sites where haplotypes 2k and 2k+1 differ (infer.py:77)."""
    G = np.asarray(G)
    n = G.shape[0] // 2 * 2
    return np.count_nonzero(G[0:n:2] != G[1:n:2], axis=1).astype(np.int64)


def estimate_scaled_params(G, positions, mu, rho, Ne):
    n, S = G.shape
    if n < 2 or S == 0 or n % 2 != 0:
        return float(mu), float(rho)
    seq_len = float(positions[-1] + 1.0)
    if seq_len <= 0:
        return float(mu), float(rho)
    het = (G[0::2] != G[1::2]).sum(axis=1, dtype=np.int64)
    pi_hat = float(het.mean()) / seq_len
    if not (pi_hat > 0 and math.isfinite(pi_hat)):
        return float(mu), float(rho)
    ratio = float(rho) / max(float(mu), 1e-30)
    return float(pi_hat / (4.0 * float(Ne))), float(pi_hat * ratio / (4.0 * float(Ne)))


def filter_segregating(G, positions):
    n = G.shape[0]
    ac = G.sum(axis=0, dtype=np.int64)
    keep = (ac > 0) & (ac < n)
    if bool(keep.all()):
        return G, positions, keep
    return np.ascontiguousarray(G[:, keep]), np.ascontiguousarray(positions[keep]), keep


def gpu_bytes_per_pair_site(mean_only):
    return 4 * (2 + (1 if mean_only else 3))


def estimate_block_gpu_bytes(core, flank, n_pairs, mean_only, n_sites=None):
    padded = core + 2 * flank
    if n_sites is not None:
        padded = min(padded, n_sites)
    return gpu_bytes_per_pair_site(mean_only) * padded * n_pairs


def recommend_core_block_size(n_sites, n_pairs, mean_only, flank, free_bytes,
                              headroom_fraction=0.20, min_headroom_bytes=512 * 1024 * 1024,
                              min_block=1024, max_block=32768):
    if n_pairs <= 0:
        return min(n_sites, max_block), 0
    bps = gpu_bytes_per_pair_site(mean_only)
    headroom = max(min_headroom_bytes, int(free_bytes * headroom_fraction))
    budget = max(0, free_bytes - headroom)
    core_max = budget // (bps * n_pairs) - 2 * flank
    if core_max <= 0:
        chosen = min(n_sites, min_block)
    elif core_max >= n_sites:
        chosen = n_sites
    else:
        chosen = max(min_block, min(1 << int(math.log2(core_max)), max_block, n_sites))
    return chosen, estimate_block_gpu_bytes(chosen, flank, n_pairs, mean_only)


def make_block_windows(S, core, flank):
    """(core_start, core_stop, padded_start, padded_stop) rows, src/bindings.cpp:2517-2534."""
    rows = []
    for cs in range(0, S, core):
        ce = min(S, cs + core)
        rows.append((cs, ce, max(0, cs - flank), min(S, ce + flank)))
    return np.array(rows, dtype=np.int32).reshape(-1, 4)


# -------------------------------------------------------------------- scan --

def fb_window(packed, positions, w0, wlen, pi, pj, Ne, tables, ci=False,
              posterior=False, n_threads=0):
    """One window of the cached FB scan; returns window-local [wlen, P] arrays."""
    packed = np.ascontiguousarray(packed, np.uint64)
    positions = np.ascontiguousarray(positions, np.float64)
    pi = np.ascontiguousarray(pi, np.int32)
    pj = np.ascontiguousarray(pj, np.int32)
    P = len(pi)
    out = {"mean": np.empty((wlen, P), np.float32)}
    if ci:
        out["lower"] = np.empty((wlen, P), np.float32)
        out["upper"] = np.empty((wlen, P), np.float32)
    if posterior:
        out["posterior_alpha"] = np.empty((wlen, P), np.float32)
        out["posterior_beta"] = np.empty((wlen, P), np.float32)
    if P == 0 or wlen == 0:
        return out
    rc = lib().oracle_fb_window(
        _ptr(packed, _u64p), packed.shape[1], _ptr(positions, _f64p), len(positions),
        int(w0), int(wlen), _ptr(pi, _i32p), _ptr(pj, _i32p), P, float(np.float32(Ne)),
        _ptr(tables, _f32p), tables.shape[1],
        _ptr(out["mean"], _f32p), _ptr(out.get("lower"), _f32p), _ptr(out.get("upper"), _f32p),
        _ptr(out.get("posterior_alpha"), _f32p), _ptr(out.get("posterior_beta"), _f32p),
        int(n_threads))
    if rc != 0:
        raise ValueError("oracle_fb_window: bad window")
    return out


def run_fb(G, positions, pairs, Ne, mu, rho, flow_field_path, mean_only=True,
           return_posterior=False, n_threads=0):
    """FlowContext(...).run_fb(...) on the CPU (src/bindings.cpp:2897-2989)."""
    S = G.shape[1]
    tables = tables_for(flow_field_path, Ne, mu, rho)
    packed = bitpack(G)
    pi = np.array([p[0] for p in pairs], np.int32)
    pj = np.array([p[1] for p in pairs], np.int32)
    return fb_window(packed, positions, 0, S, pi, pj, Ne, tables, ci=not mean_only,
                     posterior=return_posterior, n_threads=n_threads)


def run_fb_blockwise(G, positions, pairs, Ne, mu, rho, flow_field_path,
                     core_block_sites=8192, flank_sites=2048, mean_only=True,
                     return_posterior=False, n_threads=0):
    """FlowContext(...).run_fb_blockwise(...) on the CPU: every padded window
    restarts at (0, 0) and only its core rows are kept (src/bindings.cpp:2991-3345).
    Pair chunking and streams do not change the result, so they are not modelled."""
    S = G.shape[1]
    P = len(pairs)
    blocks = make_block_windows(S, core_block_sites, flank_sites)
    tables = tables_for(flow_field_path, Ne, mu, rho)
    packed = bitpack(G)
    pi = np.array([p[0] for p in pairs], np.int32)
    pj = np.array([p[1] for p in pairs], np.int32)
    keys = ["mean"] + (["lower", "upper"] if not mean_only else []) + \
        (["posterior_alpha", "posterior_beta"] if return_posterior else [])
    out = {k: np.empty((S, P), np.float32) for k in keys}
    for cs, ce, ps, pe in blocks:
        if P == 0:
            break
        w = fb_window(packed, positions, ps, pe - ps, pi, pj, Ne, tables,
                      ci=not mean_only, posterior=return_posterior, n_threads=n_threads)
        for k in keys:
            out[k][cs:ce] = w[k][cs - ps:ce - ps]
    out["blocks"] = blocks
    return out


def infer(G_or_ts, positions=None, mu=1.25e-8, rho=1e-8, Ne=10000, pairs=None,
          flow_field_path=None, mean_only=True, return_posterior=False,
          auto_estimate_theta=True, n_threads=0):
    """Oracle of gamma_smc_cu.infer (python/gamma_smc_cu/infer.py:217-296)."""
    G, positions = coerce_inputs(G_or_ts, positions)
    G, positions, _ = filter_segregating(G, positions)
    pairs = all_pairs(G.shape[0]) if pairs is None else [(int(i), int(j)) for i, j in pairs]
    if auto_estimate_theta:
        kmu, krho = estimate_scaled_params(G, positions, mu, rho, Ne)
    else:
        kmu, krho = float(mu), float(rho)
    r = run_fb(G, positions, pairs, float(Ne), kmu, krho, flow_field_path, mean_only,
               return_posterior, n_threads)
    r["pairs"] = pairs
    r["positions"] = positions
    return r


def infer_blockwise(G_or_ts, positions=None, mu=1.25e-8, rho=1e-8, Ne=10000, pairs=None,
                    flow_field_path=None, mean_only=True, core_block_sites=8192,
                    flank_sites=2048, return_posterior=False, auto_estimate_theta=True,
                    n_threads=0):
    """Oracle of gamma_smc_cu.infer_blockwise with an explicit integer block size."""
    G, positions = coerce_inputs(G_or_ts, positions)
    G, positions, _ = filter_segregating(G, positions)
    pairs = [(int(i), int(j)) for i, j in pairs]
    if auto_estimate_theta:
        kmu, krho = estimate_scaled_params(G, positions, mu, rho, Ne)
    else:
        kmu, krho = float(mu), float(rho)
    r = run_fb_blockwise(G, positions, pairs, float(Ne), kmu, krho, flow_field_path,
                         int(core_block_sites), int(flank_sites), mean_only,
                         return_posterior, n_threads)
    r["pairs"] = pairs
    r["positions"] = positions
    return r


def run_fb_summary(G, positions, pairs, Ne, mu, rho, flow_field_path, core_block_sites=0,
                   flank_sites=2048, n_threads=0):
    """Per-site mean / min / max over pairs of the posterior mean
    (FlowContext.run_fb_summary, src/bindings.cpp:2695-2788): the per-pair
    means of the full-sequence (or blockwise) scan, averaged in float64."""
    S = G.shape[1]
    if core_block_sites and 0 < core_block_sites < S:
        r = run_fb_blockwise(G, positions, pairs, Ne, mu, rho, flow_field_path,
                             core_block_sites, flank_sites, True, False, n_threads)
    else:
        r = run_fb(G, positions, pairs, Ne, mu, rho, flow_field_path, True, False, n_threads)
    m = r["mean"]
    return {"site_mean": (m.astype(np.float64).sum(axis=1) / m.shape[1]).astype(np.float32),
            "site_min": m.min(axis=1), "site_max": m.max(axis=1), "n_pairs": m.shape[1]}


def run_fwd(G, positions, pairs, Ne, mu, rho, flow_field_path, mean_only=True, n_threads=0):
    """FlowContext(...).run_fwd(...) on the CPU: the forward-only filtered
    posterior of src/kernels/gamma_smc_flow.cu:1136-1256 on the hom
    multi-step table rounded through float16 (src/bindings.cpp:2098-2107)."""
    S = G.shape[1]
    T = tables_for(flow_field_path, Ne, mu, rho)
    hom_m = np.ascontiguousarray(T[2].astype(np.float16).astype(np.float32))
    hom_c = np.ascontiguousarray(T[3].astype(np.float16).astype(np.float32))
    packed = bitpack(G)
    pi = np.ascontiguousarray([p[0] for p in pairs], np.int32)
    pj = np.ascontiguousarray([p[1] for p in pairs], np.int32)
    P = len(pi)
    positions = np.ascontiguousarray(positions, np.float64)
    out = {"mean": np.empty((S, P), np.float32)}
    if not mean_only:
        out["lower"] = np.empty((S, P), np.float32)
        out["upper"] = np.empty((S, P), np.float32)
    if P == 0 or S == 0:
        return out
    lib().oracle_fwd_only(
        _ptr(packed, _u64p), packed.shape[1], _ptr(positions, _f64p), S, _ptr(pi, _i32p),
        _ptr(pj, _i32p), P, float(np.float32(2.0 * np.float32(Ne))), _ptr(hom_m, _f32p),
        _ptr(hom_c, _f32p), hom_m.shape[0], _ptr(out["mean"], _f32p),
        _ptr(out.get("lower"), _f32p), _ptr(out.get("upper"), _f32p), int(n_threads))
    return out


def flow_fb(G, positions, pairs, Ne, mu, rho, flow_field_path, mean_only=False, n_threads=0):
    """gamma_smc_cu.gamma_smc_flow_fb on the CPU: the uncached flow-field FB
    (src/kernels/gamma_smc_flow.cu:29-163, 168-398) with the launcher's float
    rates (:342-344) and no theta calibration."""
    S = G.shape[1]
    u, v, _ = load_flow_field(flow_field_path)
    u = np.ascontiguousarray(u, np.float32).ravel()
    v = np.ascontiguousarray(v, np.float32).ravel()
    ne, fmu, frho = np.float32(Ne), np.float32(mu), np.float32(rho)
    lam = np.float32(1.0) / (np.float32(2.0) * ne)
    srho = np.float32(4.0) * ne * frho
    smu = np.float32(2.0) * fmu / lam
    packed = bitpack(G)
    pi = np.ascontiguousarray([p[0] for p in pairs], np.int32)
    pj = np.ascontiguousarray([p[1] for p in pairs], np.int32)
    P = len(pi)
    positions = np.ascontiguousarray(positions, np.float64)
    out = {"mean": np.empty((S, P), np.float32)}
    if not mean_only:
        out["lower"] = np.empty((S, P), np.float32)
        out["upper"] = np.empty((S, P), np.float32)
    if P == 0 or S == 0:
        return out
    lib().oracle_flow_fb(_ptr(packed, _u64p), packed.shape[1], _ptr(positions, _f64p), S,
                         _ptr(pi, _i32p), _ptr(pj, _i32p), P, _ptr(u, _f32p), _ptr(v, _f32p),
                         float(srho), float(smu), float(ne), _ptr(out["mean"], _f32p),
                         _ptr(out.get("lower"), _f32p), _ptr(out.get("upper"), _f32p),
                         int(n_threads))
    return out
