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
