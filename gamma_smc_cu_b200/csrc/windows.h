// Blockwise windows: core [cs, ce) with flanks, padded window [ps, pe).
//
// The reference cuts the sites into cores of core_block_sites and pads each
// with flank_sites on both sides, clamped to the sequence
// (src/bindings.cpp:2517-2534).  The arithmetic is int64 throughout and core
// and flank are clamped to the sequence length first, so any non-negative
// int64 input (a flank of 2^40 meaning "the whole sequence") gives bounds in
// [0, n_sites].  Header-only so host planning, device kernels and a plain C++
// test share one definition.
#pragma once

#include <stdint.h>

#include <cmath>

#if defined(__CUDACC__)
#define GSMC_HD __host__ __device__ __forceinline__
#else
#define GSMC_HD inline
#endif

namespace gsmc {

struct WindowBounds {
  int64_t ps, cs, ce, pe;
};

// Core length actually used: at least 1, at most n_sites (a core longer than
// the sequence is the whole sequence).
GSMC_HD int64_t clamp_core(int64_t core_block_sites, int64_t n_sites) {
  const int64_t s = n_sites > 1 ? n_sites : 1;
  return core_block_sites < 1 ? 1 : (core_block_sites > s ? s : core_block_sites);
}

// Flank length actually used: in [0, n_sites] (a longer flank reaches the
// sequence ends either way).
GSMC_HD int64_t clamp_flank(int64_t flank_sites, int64_t n_sites) {
  const int64_t s = n_sites > 0 ? n_sites : 0;
  return flank_sites < 0 ? 0 : (flank_sites > s ? s : flank_sites);
}

// Number of windows of n_sites >= 0 sites with cores of core_block_sites.
GSMC_HD int64_t window_count(int64_t n_sites, int64_t core_block_sites) {
  if (n_sites <= 0) return 0;
  const int64_t core = clamp_core(core_block_sites, n_sites);
  return (n_sites - 1) / core + 1;
}

// Window w (0 <= w < window_count) of n_sites sites.
GSMC_HD WindowBounds window_bounds(int64_t w, int64_t n_sites, int64_t core_block_sites,
                                   int64_t flank_sites) {
  const int64_t core = clamp_core(core_block_sites, n_sites);
  const int64_t flank = clamp_flank(flank_sites, n_sites);
  WindowBounds b;
  b.cs = w * core;
  b.ce = b.cs + core < n_sites ? b.cs + core : n_sites;
  b.ps = b.cs - flank > 0 ? b.cs - flank : 0;
  b.pe = b.ce + flank < n_sites ? b.ce + flank : n_sites;
  return b;
}

// Cut points cut[0] = cs < cut[1] < ... < cut[K] = ce of the core of window
// [ps, pe) into K >= 1 speculative chunks of equal cost (host only).  Chunk
// k runs forward from cut[k] - pre_k to cut[k+1] and backward from
// cut[k+1] + post_k to cut[k], where pre_0 = cs - ps (the window's own left
// flank), pre_k = flank otherwise, post_(K-1) = pe - ce and post_k = flank
// otherwise.  A core site costs core_weight burn-in sites (its forward step
// also stores the state, its backward step reads it back and combines), so
// chunk k costs 2 w len_k + pre_k + post_k.  Equal cost T gives
// len_k = (T - pre_k - post_k) / (2 w): a chunk at an end of the sequence,
// where the window has no flank, takes the cost of the burn-in it does not
// run as extra core.  Equal lengths when a chunk would come out shorter than
// one flank (or than one site).
inline void chunk_cuts(int64_t ps, int64_t cs, int64_t ce, int64_t pe, int K, int64_t flank,
                       double core_weight, int64_t* cut) {
  const int64_t len = ce - cs;
  for (int k = 0; k <= K; ++k) cut[k] = cs + len * k / K;
  if (K <= 1) return;
  const double w = core_weight > 0.0 ? core_weight : 1.0;
  const double e0 = (double)(cs - ps), e1 = (double)(pe - ce), f = (double)flank;
  const double T = (2.0 * w * (double)len + e0 + e1 + 2.0 * (K - 1) * f) / K;
  const int64_t min_len = flank > 1 ? flank : 1;
  double acc = 0.0;
  int64_t prev = cs;
  for (int k = 0; k < K; ++k) {
    const double pre = k == 0 ? e0 : f, post = k == K - 1 ? e1 : f;
    acc += (T - pre - post) / (2.0 * w);
    const int64_t next = k == K - 1 ? ce : cs + (int64_t)std::llround(acc);
    if (next - prev < min_len) {
      for (int j = 0; j <= K; ++j) cut[j] = cs + len * j / K;
      return;
    }
    cut[k + 1] = next;
    prev = next;
  }
}

}  // namespace gsmc
