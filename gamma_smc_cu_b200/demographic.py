"""Flow-field generation (on the GPU, float64) and demography-aware contexts.

Same public functions as the reference's ``gamma_smc_cu.demographic``
(python/gamma_smc_cu/demographic.py:146-286): ``generate_flow_field``,
``write_flow_field``, ``load_flow_field``, ``estimate_demography`` and
``DemographicFlowContext``.  The per-cell fits of ``generate_flow_field`` run
as one CUDA block per grid cell (``gsmc_generate_flow_field``); the grid
set-up, the epoch bookkeeping and the file formats are the reference's.
"""
from __future__ import annotations

import os
import tempfile

import numpy as np

from . import _lib
from ._lib import check, ptr

_CALIBRATION_FACTOR = 5.302  # demographic.py:14


def _grid(mean_min, mean_max, cv_min, cv_max, mean_n, cv_n):
    """Gamma (alpha, beta) of every cell, as demographic.py:169-183 derives them."""
    log10_mean = np.linspace(np.log10(mean_min), np.log10(mean_max), mean_n)
    log10_cv = np.linspace(np.log10(cv_min), np.log10(cv_max), cv_n)
    mean = 10.0 ** log10_mean[:, None] * np.ones((1, cv_n))
    cv = 10.0 ** log10_cv[None, :] * np.ones((mean_n, 1))
    std = cv * mean
    alpha = (mean / std) ** 2
    beta = mean / std ** 2
    return np.ascontiguousarray(alpha), np.ascontiguousarray(beta)


def _epochs(Ne_values, epoch_boundaries, Ne_ref):
    """(start, rate, cumulative rate) per epoch in scaled time (demographic.py:150-158)."""
    M = len(Ne_values)
    scale = 2.0 * Ne_ref
    t_b = np.zeros(M + 1)
    t_b[1:M] = np.array(epoch_boundaries[1:M], dtype=np.float64) / scale
    lam_v = Ne_ref / np.array(Ne_values, dtype=np.float64)
    L_b = np.zeros(M + 1)
    for k in range(1, M):
        L_b[k] = L_b[k - 1] + lam_v[k - 1] * (t_b[k] - t_b[k - 1])
    return (np.ascontiguousarray(t_b[:M]), np.ascontiguousarray(lam_v),
            np.ascontiguousarray(L_b[:M]))


def generate_flow_field(Ne_values=None, epoch_boundaries=None, Ne_ref=10000,
                        mean_min=1e-5, mean_max=1e2, cv_min=1e-2, cv_max=1.0,
                        mean_n=51, cv_n=50, n_steps=500, verbose=True):
    """(u, v) [mean_n, cv_n] float64 flow field; constant Ne unless
    ``Ne_values`` / ``epoch_boundaries`` give a piecewise-constant history."""
    alpha, beta = _grid(mean_min, mean_max, cv_min, cv_max, mean_n, cv_n)
    u = np.zeros((mean_n, cv_n))
    v = np.zeros((mean_n, cv_n))
    if Ne_values is not None:
        start, rate, cum = _epochs(Ne_values, epoch_boundaries, Ne_ref)
        n_ep = len(start)
    else:
        start = rate = cum = None
        n_ep = 0
    check(_lib.load().gsmc_generate_flow_field(
        ptr(alpha, _lib.c_f64p), ptr(beta, _lib.c_f64p), int(mean_n), int(cv_n), int(n_steps),
        n_ep, ptr(start, _lib.c_f64p), ptr(rate, _lib.c_f64p), ptr(cum, _lib.c_f64p),
        float(_CALIBRATION_FACTOR), ptr(u, _lib.c_f64p), ptr(v, _lib.c_f64p)))
    if verbose:
        print(f"  flow field: {mean_n * cv_n}/{mean_n * cv_n} (GPU)", flush=True)
    return u, v


def write_flow_field(path, u, v, mean_min=1e-5, mean_max=1e2, cv_min=1e-2, cv_max=1.0):
    """Text format read by the context: two header lines, then u, then v
    (demographic.py:215-220)."""
    mn, cn = u.shape
    with open(path, "w") as f:
        f.write(f"{mean_min} {mean_max} {mn}\n{cv_min} {cv_max} {cn}\n")
        for row in u:
            f.write(" ".join(f"{x:.10f}" for x in row) + "\n")
        for row in v:
            f.write(" ".join(f"{x:.10f}" for x in row) + "\n")


def load_flow_field(path):
    """(u, v, mean_min, mean_max, cv_min, cv_max) of a flow-field file."""
    with open(path) as f:
        parts = f.read().split()
    i = 0
    mm, mx, mn = float(parts[i]), float(parts[i + 1]), int(parts[i + 2])
    i += 3
    cm, cx, cn = float(parts[i]), float(parts[i + 1]), int(parts[i + 2])
    i += 3
    u = np.array([float(x) for x in parts[i:i + mn * cn]]).reshape(mn, cn)
    i += mn * cn
    v = np.array([float(x) for x in parts[i:i + mn * cn]]).reshape(mn, cn)
    return u, v, mm, mx, cm, cx


def estimate_demography(tmrca_means, Ne_init, n_epochs=20, t_max=None):
    """Piecewise-constant Ne from posterior TMRCA means (demographic.py:222-247).

    Epoch edges are quadratic in [0, t_max] (default 10 Ne_init).  An epoch
    with at least 10 means, a positive width and more than 1% of the means
    surviving to its start gets Ne = max(100, 1 / (2 * hazard)), hazard = the
    epoch's density over the surviving fraction; the others keep Ne_init.
    Returns (Ne values, epoch boundaries).
    """
    if t_max is None:
        t_max = 10.0 * Ne_init
    vals = np.asarray(tmrca_means, dtype=np.float64).ravel()
    vals = np.sort(vals[np.isfinite(vals) & (vals > 0)])
    edges = t_max * np.linspace(0, 1, n_epochs + 1) ** 2
    edges[0] = 0.0
    n = len(vals)
    at_or_above = n - np.searchsorted(vals, edges, side="left")   # #(vals >= edge)
    counts = at_or_above[:-1] - at_or_above[1:]                   # #(lo <= vals < hi)
    widths = np.diff(edges)
    Ne_values = np.full(n_epochs, Ne_init, dtype=np.float64)
    for k in np.flatnonzero((counts >= 10) & (widths > 0)):
        density = counts[k] / (n * widths[k])
        survival = at_or_above[k] / n
        if survival > 0.01:
            Ne_values[k] = max(100.0, 1.0 / (2.0 * density / survival))
    return Ne_values, edges


class DemographicFlowContext:
    """Two-stage context (demographic.py:249-286): decode calibration pairs
    with the given flow field, estimate N(t) from their means, generate the
    demographic flow field on the GPU, and keep a context on it."""

    def __init__(self, G, positions, Ne_init, mu, rho, flow_field_path,
                 n_calibration_pairs=50, n_epochs=20, n_steps=500,
                 cache_steps=0, gpu_id=0, verbose=True):
        import time

        from . import _core
        self.S = len(positions)
        self.Ne_init = Ne_init
        n = G.shape[0]
        _core.set_device(gpu_id)
        if verbose:
            print("Stage 1: estimating demography...", flush=True)
        rng = np.random.default_rng(42)
        n_cal = min(n_calibration_pairs, n * (n - 1) // 2)
        cs = set()
        while len(cs) < n_cal:
            a, b = sorted(rng.choice(n, 2, replace=False))
            cs.add((int(a), int(b)))
        ctx = _core.FlowContext(G, positions, float(Ne_init), mu, rho, flow_field_path,
                                cache_steps)
        r = ctx.run_fb(sorted(cs), mean_only=True)
        ctx.close()
        self.Ne_values, self.epoch_boundaries = estimate_demography(r["mean"], Ne_init,
                                                                    n_epochs=n_epochs)
        if verbose:
            print(f"  N(t): {self.Ne_values[:3].astype(int)} ... "
                  f"{self.Ne_values[-2:].astype(int)}", flush=True)
            print("Stage 2: generating demographic flow field...", flush=True)
        t0 = time.perf_counter()
        u, v = generate_flow_field(Ne_values=self.Ne_values,
                                   epoch_boundaries=self.epoch_boundaries, Ne_ref=Ne_init,
                                   n_steps=n_steps, verbose=verbose)
        if verbose:
            print(f"  done in {time.perf_counter() - t0:.1f}s", flush=True)
        self._ff_dir = tempfile.mkdtemp()
        self._ff_path = os.path.join(self._ff_dir, "d.txt")
        write_flow_field(self._ff_path, u, v)
        self.ctx = _core.FlowContext(G, positions, float(Ne_init), mu, rho, self._ff_path,
                                     cache_steps)
        if verbose:
            print("Ready.", flush=True)

    def run_fb(self, pairs, mean_only=True):
        return self.ctx.run_fb(pairs, mean_only)

    def run_fwd(self, pairs, mean_only=True):
        return self.ctx.run_fwd(pairs, mean_only)

    def run_fb_summary(self, pairs):
        return self.ctx.run_fb_summary(pairs)

    @property
    def device_id(self):
        return self.ctx.device_id

    @property
    def demography(self):
        return self.Ne_values.copy(), self.epoch_boundaries.copy()

    def __del__(self):
        try:
            if hasattr(self, "_ff_path") and os.path.exists(self._ff_path):
                os.unlink(self._ff_path)
            if hasattr(self, "_ff_dir") and os.path.exists(self._ff_dir):
                os.rmdir(self._ff_dir)
        except OSError:
            pass
