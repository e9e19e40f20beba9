"""Seeded synthetic haplotype data with the shapes of the benchmark cohorts.

msprime is not available, so coalescent simulations are replaced by a
Li-Stephens-style copying mosaic: ``n_founders`` founder haplotypes carry
derived alleles with a 1/k site-frequency spectrum, every haplotype copies a
founder and switches to a random founder at rate ``switch_rate`` per base
pair, and private mutations flip a small fraction of alleles.  Pairs that copy
the same founder share long identical tracts, pairs that copy different
founders differ at founder-polymorphic sites, which gives het/hom runs like
those of real data.  Every site is made segregating.

Positions are strictly increasing integers with i.i.d. exponential gaps
(mean span / n_sites, rounded, at least 1 bp).  The default span is the
neutral expectation for n_sites segregating sites: n_sites / (4 Ne mu H_{n-1}).

Named cohorts (sizes as in the benchmark configurations):

* ``small``  40 haplotypes, 2,127 sites over 1 Mb, all 780 pairs (seeds 1/2)
* ``chrom``  356 haplotypes, 400,000 sites, 63,190 pairs (seeds 3/4)
* ``cohort`` 2,000 haplotypes, 200,000 sites, 1,000,000 random pairs (seeds 7/8/9)
"""
from __future__ import annotations

import math

import numpy as np


def harmonic(n):
    return float(np.sum(1.0 / np.arange(1, n)))


def neutral_span(n_haps, n_sites, Ne=1e4, mu=1.25e-8):
    return n_sites / (4.0 * Ne * mu * harmonic(n_haps))


def positions_for(n_sites, span_bp, seed):
    rng = np.random.default_rng(seed)
    gaps = np.maximum(1, np.rint(rng.exponential(span_bp / max(n_sites, 1), n_sites)))
    return (np.cumsum(gaps) - 1.0).astype(np.float64)


def haplotypes(n_haps, positions, seed, n_founders=24, switch_rate=2e-5, private_rate=2e-3,
               chunk=64):
    """[n_haps, n_sites] uint8 mosaic genotypes (see module docstring)."""
    S = len(positions)
    rng = np.random.default_rng(seed)
    K = n_founders
    # founder alleles: derived count k in [1, K-1] with weight 1/k
    w = 1.0 / np.arange(1, K)
    k = rng.choice(np.arange(1, K), size=S, p=w / w.sum())
    keys = rng.random((S, K))
    ranks = np.argsort(np.argsort(keys, axis=1), axis=1)
    founders = (ranks < k[:, None]).astype(np.uint8).T.copy()  # [K, S]
    gaps = np.diff(positions, prepend=positions[0] - 1.0) if S else np.zeros(0)
    p_switch = -np.expm1(-switch_rate * gaps)
    G = np.empty((n_haps, S), np.uint8)
    cols = np.arange(S)
    for h0 in range(0, n_haps, chunk):
        h1 = min(n_haps, h0 + chunk)
        hc = h1 - h0
        sw = rng.random((hc, S)) < p_switch[None, :]
        if S:
            sw[:, 0] = True
        ids = rng.integers(0, K, size=(hc, S), dtype=np.int64)
        last = np.where(sw, cols[None, :], 0)
        np.maximum.accumulate(last, axis=1, out=last)
        fidx = np.take_along_axis(ids, last, axis=1)
        g = founders[fidx, cols[None, :]]
        g ^= (rng.random((hc, S)) < private_rate).astype(np.uint8)
        G[h0:h1] = g
    # every site segregating: fix all-0 / all-1 columns with one flipped allele
    ac = G.sum(axis=0, dtype=np.int64)
    for s in np.flatnonzero(ac == 0):
        G[rng.integers(n_haps), s] = 1
    for s in np.flatnonzero(ac == n_haps):
        G[rng.integers(n_haps), s] = 0
    return G


def all_pairs(n):
    """All (i, j), i > j, row-major: pair index i(i-1)/2 + j."""
    i, j = np.tril_indices(n, -1)
    return np.stack([i, j], axis=1).astype(np.int32)


def pairs_from_index(idx):
    """Vectorised inverse of i(i-1)/2 + j for i > j."""
    idx = np.asarray(idx, np.int64)
    i = np.floor((1.0 + np.sqrt(1.0 + 8.0 * idx.astype(np.float64))) / 2.0).astype(np.int64)
    i -= (i * (i - 1) // 2 > idx)
    i += ((i + 1) * i // 2 <= idx)
    j = idx - i * (i - 1) // 2
    return np.stack([i, j], axis=1).astype(np.int32)


def random_pairs(n_haps, n_pairs, seed):
    """n_pairs distinct pairs drawn uniformly, in pair-index order."""
    total = n_haps * (n_haps - 1) // 2
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(total, size=min(n_pairs, total), replace=False))
    return pairs_from_index(idx)


COHORTS = {
    # name: (n_haps, n_sites, span_bp or None, seed_positions, seed_genotypes)
    "small": (40, 2127, 1.0e6, 1, 2),
    "chrom": (356, 400_000, None, 3, 4),
    "cohort": (2000, 200_000, None, 7, 8),
}


def cohort(name, n_sites=None):
    """(G, positions) of a named cohort; n_sites truncates to a prefix."""
    n, S, span, sp, sg = COHORTS[name]
    span = neutral_span(n, S) if span is None else span
    pos = positions_for(S, span, sp)
    if n_sites is not None:
        pos = pos[:n_sites]
    return haplotypes(n, pos, sg), pos


def _log_uniform_int(rng, lo, hi, size=None):
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size))).astype(np.int64)


def _distinct_pairs(rng, n_haps, n):
    total = n_haps * (n_haps - 1) // 2
    return pairs_from_index(np.sort(rng.choice(total, size=min(n, total), replace=False)))


def job_mix(n_haps, n_sites, n_jobs=512, seed=5, pairs_range=(1, 4096),
            window_range=(1_000, 200_000)):
    """Uneven batch of jobs: pair count log-uniform in pairs_range (random
    distinct pairs), window length in sites log-uniform in window_range at a
    uniform random start; both clamped to the cohort.  Returns dicts with
    pairs / site_begin / site_end (mean_only)."""
    rng = np.random.default_rng(seed)
    n_p = _log_uniform_int(rng, pairs_range[0], pairs_range[1], n_jobs)
    n_w = _log_uniform_int(rng, window_range[0], window_range[1], n_jobs)
    jobs = []
    for p, w in zip(n_p, n_w):
        w = int(min(max(1, w), n_sites))
        s0 = int(rng.integers(0, n_sites - w + 1))
        jobs.append({"pairs": _distinct_pairs(rng, n_haps, int(max(1, p))), "site_begin": s0,
                     "site_end": s0 + w})
    return jobs


def job_mix_bp(positions, n_haps, n_jobs=512, seed=5, pairs_range=(1, 4096),
               window_bp=(1_000, 200_000)):
    """job_mix with window lengths in base pairs: each window is log-uniform
    in window_bp at a uniform start and covers the sites inside it (at least
    one); pair counts as in job_mix, clamped to the cohort's pairs."""
    rng = np.random.default_rng(seed)
    positions = np.asarray(positions, np.float64)
    n_p = _log_uniform_int(rng, pairs_range[0], pairs_range[1], n_jobs)
    lo, hi = float(positions[0]), float(positions[-1]) + 1.0
    jobs = []
    for p in n_p:
        length = float(min(hi - lo, np.exp(rng.uniform(np.log(window_bp[0]), np.log(window_bp[1])))))
        a = float(rng.uniform(lo, hi - length)) if hi - length > lo else lo
        s0 = int(np.searchsorted(positions, a, side="left"))
        s1 = int(np.searchsorted(positions, a + length, side="left"))
        s0 = min(s0, len(positions) - 1)
        s1 = max(s1, s0 + 1)
        jobs.append({"pairs": _distinct_pairs(rng, n_haps, int(max(1, p))), "site_begin": s0,
                     "site_end": s1})
    return jobs


def request_stream(positions, n_haps, n_requests, rate, seed=6, pairs_range=(1, 8192),
                   region_bp=(1_000, 5_000_000), posterior_fraction=0.2):
    """Poisson stream of TMRCA queries: arrival times (s) at ``rate`` per
    second, pair subsets of log-uniform size (random distinct pairs, clamped
    to the cohort), regions of log-uniform length in base pairs at a uniform
    start (clamped to the sequence), a ``posterior_fraction`` of them asking
    for the full posterior (mean + alpha + beta), the rest mean-only.
    Returns dicts with t / pairs / region_bp / mean_only / return_posterior."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests)) if rate > 0 else np.zeros(n_requests)
    lo, hi = float(positions[0]), float(positions[-1]) + 1.0
    out = []
    for k in range(n_requests):
        n = int(max(1, _log_uniform_int(rng, pairs_range[0], pairs_range[1])))
        length = float(min(hi - lo, np.exp(rng.uniform(np.log(region_bp[0]), np.log(region_bp[1])))))
        a = float(rng.uniform(lo, hi - length)) if hi - length > lo else lo
        post = bool(rng.random() < posterior_fraction)
        out.append({"t": float(t[k]), "pairs": _distinct_pairs(rng, n_haps, n),
                    "region_bp": (a, a + length), "mean_only": True, "return_posterior": post})
    return out
