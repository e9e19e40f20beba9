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

}  // namespace gsmc
