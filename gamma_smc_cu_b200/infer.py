"""``infer`` / ``infer_blockwise``: the reference's public API over the B200 scan.

Signatures, defaults, validation messages, warnings, the auto block sizing
and the result dictionaries follow ``python/gamma_smc_cu/infer.py`` so callers
can switch packages without changes.  Device work goes through
``gamma_smc_cu_b200._core`` (looked up at call time).
"""
from __future__ import annotations

import math
import os
import warnings

import numpy as np

_F32 = 4
_MIN_BLOCK_SITES = 1024
_MAX_BLOCK_SITES = 32768
_DEFAULT_BLOCK_SITES = 8192
_PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))


def _coerce_inputs(G_or_ts, positions):
    """(G uint8 [n, S] C-contiguous, positions float64 [S]) from a tree
    sequence or a haplotype matrix (infer.py:20-41)."""
    if hasattr(G_or_ts, "genotype_matrix"):
        ts = G_or_ts
        G = ts.genotype_matrix().T.astype(np.uint8, copy=False)
        pos = np.array([site.position for site in ts.variants()], dtype=np.float64)
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


def _scaled_params_from_counts(het_per_individual, positions, mu, rho, Ne):
    """(effective_mu, effective_rho) from per-diploid het counts (infer.py:44-99).

    The scaled mutation rate is the mean per-diploid heterozygosity over the
    span [0, last position + 1); the scaled recombination rate keeps the
    user's rho/mu ratio; both are returned divided by 4 Ne so that 4 Ne * rate
    reproduces them.  The raw (mu, rho) come back for a non-positive span or
    estimate.
    """
    span = float(positions[-1] + 1.0)
    if span <= 0:
        return float(mu), float(rho)
    pi_hat = float(np.asarray(het_per_individual, np.int64).mean()) / span
    if not (pi_hat > 0 and math.isfinite(pi_hat)):
        return float(mu), float(rho)
    four_ne = 4.0 * float(Ne)
    ratio = float(rho) / max(float(mu), 1e-30)
    return float(pi_hat / four_ne), float(pi_hat * ratio / four_ne)


def _estimate_scaled_params(G, positions, mu, rho, Ne):
    """Data-driven (effective_mu, effective_rho) as gamma_smc's auto mode sets
    them (infer.py:44-99), counting on the host: haplotypes 2k and 2k+1 form
    individual k.  The raw (mu, rho) come back unchanged for n < 2, odd n, no
    sites, or a non-positive estimate.  ``infer`` makes the same counts on the
    GPU (``_core.diploid_het_counts``); both give identical int64 counts.
    """
    n, S = G.shape
    if n < 2 or S == 0 or n % 2:
        return float(mu), float(rho)
    het_per_individual = np.count_nonzero(G[0::2] != G[1::2], axis=1).astype(np.int64)
    return _scaled_params_from_counts(het_per_individual, positions, mu, rho, Ne)


def _filter_segregating(G, positions):
    """Drop sites whose allele count is 0 or n (infer.py:102-126); returns
    (G, positions, keep) and copies nothing when every site segregates."""
    counts = G.sum(axis=0, dtype=np.int64)
    keep = (counts > 0) & (counts < G.shape[0])
    if keep.all():
        return G, positions, keep
    return np.ascontiguousarray(G[:, keep]), np.ascontiguousarray(positions[keep]), keep


def _resolve_flow_field_path(flow_field_path):
    if flow_field_path is not None:
        return flow_field_path
    bundled = os.path.join(_PACKAGE_DIR, "data", "default_flow_field.txt")
    env = os.environ.get("GAMMA_SMC_FLOW_FIELD")
    for candidate in (env, bundled):
        if candidate and os.path.exists(candidate):
            return candidate
    raise FileNotFoundError("No flow field file found. Pass flow_field_path explicitly.")


def _normalize_pairs(pairs):
    return [(int(i), int(j)) for i, j in pairs]


def _gpu_bytes_per_pair_site(mean_only):
    """Memory model of the blockwise call per pair and padded site: two
    forward-state floats plus one (mean) or three (mean, lower, upper) outputs."""
    return _F32 * (2 + (1 if mean_only else 3))


def _query_free_gpu_bytes():
    try:
        from gamma_smc_cu_b200 import _core
        free_bytes, _total = _core.cuda_mem_info()
        return int(free_bytes)
    except Exception:
        return None


def _estimate_block_gpu_bytes(core_block_sites, flank_sites, n_pairs, mean_only, n_sites=None):
    padded = core_block_sites + 2 * flank_sites
    if n_sites is not None:
        padded = min(padded, n_sites)
    return _gpu_bytes_per_pair_site(mean_only) * padded * n_pairs


def _recommend_core_block_size(n_sites, n_pairs, mean_only, flank_sites, free_bytes,
                               headroom_fraction=0.20, min_headroom_bytes=512 * 1024 * 1024,
                               min_block=_MIN_BLOCK_SITES, max_block=_MAX_BLOCK_SITES):
    """Largest core block (a power of two in [min_block, max_block], or n_sites
    when everything fits) whose padded window fits all pairs in the free memory
    left after headroom (infer.py:181-214).  Returns (core, estimated bytes)."""
    if n_pairs <= 0:
        return min(n_sites, max_block), 0
    per_site = _gpu_bytes_per_pair_site(mean_only) * n_pairs
    headroom = max(min_headroom_bytes, int(free_bytes * headroom_fraction))
    core_max = max(0, free_bytes - headroom) // per_site - 2 * flank_sites
    if core_max <= 0:
        chosen = min(n_sites, min_block)
    elif core_max >= n_sites:
        chosen = n_sites
    else:
        chosen = max(min_block, min(1 << int(math.log2(core_max)), max_block, n_sites))
    return chosen, _estimate_block_gpu_bytes(chosen, flank_sites, n_pairs, mean_only)


def _scaled_rates(G, positions, mu, rho, Ne, auto_estimate_theta):
    """Rates for the context: the chromosome-wide calibration counts are made
    on the GPU from bit-packed genotypes (``_core.diploid_het_counts``,
    looked up at call time), the rest as in _estimate_scaled_params."""
    from gamma_smc_cu_b200 import _core
    if not auto_estimate_theta:
        return float(mu), float(rho)
    n, S = G.shape
    if n < 2 or S == 0 or n % 2:
        return float(mu), float(rho)
    return _scaled_params_from_counts(_core.diploid_het_counts(G), positions, mu, rho, Ne)


def infer(G_or_ts, positions=None, mu=1.25e-8, rho=1e-8, Ne=10000, pairs=None,
          flow_field_path=None, mean_only=True, return_posterior=False,
          auto_estimate_theta=True):
    """Posterior pairwise TMRCA at every segregating site.

    Returns a dict with ``mean`` ([n_sites, n_pairs] float32, generations),
    ``lower``/``upper`` (95% bounds) unless ``mean_only``, ``posterior_alpha``/
    ``posterior_beta`` (Gamma posterior in time scaled by 2 Ne) when
    ``return_posterior``, plus ``pairs`` and ``positions`` of the decoded
    (segregating) sites.  Default pairs: every (i, j) with i > j, row-major.
    """
    from gamma_smc_cu_b200 import _core

    G, positions = _coerce_inputs(G_or_ts, positions)
    G, positions, _ = _filter_segregating(G, positions)
    n = G.shape[0]
    pairs = [(i, j) for i in range(n) for j in range(i)] if pairs is None else _normalize_pairs(pairs)
    flow_field_path = _resolve_flow_field_path(flow_field_path)
    kernel_mu, kernel_rho = _scaled_rates(G, positions, mu, rho, Ne, auto_estimate_theta)
    ctx = _core.FlowContext(G, positions, float(Ne), kernel_mu, kernel_rho, flow_field_path, 0)
    result = ctx.run_fb(pairs, mean_only=mean_only, return_posterior=return_posterior)
    result["pairs"] = pairs
    result["positions"] = positions
    return result


def infer_blockwise(G_or_ts, positions=None, mu=1.25e-8, rho=1e-8, Ne=10000, pairs=None,
                    flow_field_path=None, mean_only=True, core_block_sites="auto",
                    flank_sites=2048, pair_batch_size=-1, max_streams=1, verbose=False,
                    return_posterior=False, auto_estimate_theta=True):
    """Blockwise decoding: cores of ``core_block_sites`` sites, each padded by
    ``flank_sites`` of burn-in on both sides, stitched into [n_sites, n_pairs].

    ``core_block_sites="auto"`` picks the largest power-of-two core that fits
    all pairs in free GPU memory.  The result adds ``blocks`` (int32 rows of
    core_start, core_stop, padded_start, padded_stop).
    """
    from gamma_smc_cu_b200 import _core

    if pairs is None:
        raise ValueError("infer_blockwise requires explicit pairs in v1.")
    if return_posterior and max_streams > 1:
        raise ValueError(
            "infer_blockwise: return_posterior=True is currently only supported with "
            "max_streams=1. Run blockwise posterior decoding in single-stream mode.")
    if flank_sites < 0:
        raise ValueError("flank_sites must be non-negative.")
    if pair_batch_size == 0 or pair_batch_size < -1:
        raise ValueError("pair_batch_size must be positive or -1 for auto.")
    if max_streams <= 0:
        raise ValueError("max_streams must be positive.")
    auto_block = core_block_sites in ("auto", None)
    if not auto_block:
        if not isinstance(core_block_sites, (int, np.integer)):
            raise TypeError("core_block_sites must be int or 'auto', got "
                            f"{type(core_block_sites).__name__}.")
        if core_block_sites <= 0:
            raise ValueError("core_block_sites must be positive (or 'auto').")

    G, positions = _coerce_inputs(G_or_ts, positions)
    G, positions, _ = _filter_segregating(G, positions)
    pairs = _normalize_pairs(pairs)
    n_sites = G.shape[1]
    n_pairs = len(pairs)

    free_bytes = _query_free_gpu_bytes()
    if auto_block:
        if free_bytes is None:
            warnings.warn(
                "infer_blockwise(core_block_sites='auto') could not query GPU memory; "
                f"falling back to core_block_sites={_DEFAULT_BLOCK_SITES}.", stacklevel=2)
            core_block_sites = _DEFAULT_BLOCK_SITES
        else:
            core_block_sites, est = _recommend_core_block_size(
                n_sites, n_pairs, mean_only, flank_sites, free_bytes)
            if verbose:
                print(f"[infer_blockwise] auto core_block_sites={core_block_sites} "
                      f"(free_gpu={free_bytes / 1e9:.2f}GB, est_block={est / 1e9:.2f}GB, "
                      f"n_blocks={max(1, math.ceil(n_sites / core_block_sites))})", flush=True)
    elif free_bytes is not None and n_pairs > 0:
        est = _estimate_block_gpu_bytes(core_block_sites, flank_sites, n_pairs, mean_only,
                                        n_sites=n_sites)
        if est > free_bytes:
            suggested, _ = _recommend_core_block_size(n_sites, n_pairs, mean_only, flank_sites,
                                                      free_bytes)
            warnings.warn(
                f"infer_blockwise: core_block_sites={core_block_sites} with "
                f"flank_sites={flank_sites} for {n_pairs} pairs needs ~{est / 1e9:.2f}GB GPU "
                f"memory but only {free_bytes / 1e9:.2f}GB is free. The backend will fall "
                f"back to chunking pairs (slower). Suggested: core_block_sites={suggested} "
                "(or pass 'auto').", stacklevel=2)

    if flank_sites == 0 and core_block_sites < n_sites:
        raise ValueError(
            "infer_blockwise: flank_sites=0 with core_block_sites < n_sites "
            f"(core_block_sites={core_block_sites}, n_sites={n_sites}) produces invalid "
            "results because each block restarts the forward/backward pass from the "
            "marginal prior with no warm-up history. Pass flank_sites>=256 (default 2048) "
            "or set core_block_sites>=n_sites to decode the whole sequence as a single block.")

    # -1 means "auto" in the backend; cap it by the actual pair count so the
    # backend never sizes buffers for more pairs than it has.
    batch = max(1, n_pairs) if pair_batch_size == -1 else pair_batch_size

    flow_field_path = _resolve_flow_field_path(flow_field_path)
    kernel_mu, kernel_rho = _scaled_rates(G, positions, mu, rho, Ne, auto_estimate_theta)
    ctx = _core.FlowContext(G, positions, float(Ne), kernel_mu, kernel_rho, flow_field_path, 0)
    result = ctx.run_fb_blockwise(pairs, core_block_sites=int(core_block_sites),
                                  flank_sites=flank_sites, pair_batch_size=batch,
                                  max_streams=max_streams, mean_only=mean_only,
                                  return_posterior=return_posterior)
    result["pairs"] = pairs
    result["positions"] = positions
    return result
