// Launch planning arithmetic of the scan: how many exact speculative chunks
// a window is cut into, given the launch's tasks and the resident tiles.
//
// Host-only and free of CUDA types, so the context (capi.cu) and a plain C++
// test share one definition.  Every number here only decides how work is
// split; the chunked decode is bit-identical to the whole-window one.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <vector>

namespace gsmc {
namespace plan {

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Estimated duration, in pair-steps of one tile, of a persistent launch of n
// equal tasks of `steps` pair-steps each on r resident tiles: full waves of r
// tasks plus a partial wave of fraction f.  A partial wave runs faster than
// its share of the GPU (fewer CTAs share the SMs) and, after full waves,
// overlaps their uneven ends; fitted on the 50,000-site full-posterior slice
// (63,190 pairs, 1,184 resident tiles, 2 to 8 chunks): alone it costs
// 0.3 + 0.64 f of a full wave, after full waves 0.26 + 0.37 f.
inline double launch_cost(int64_t n, int64_t r, double steps) {
  if (n <= 0 || r <= 0) return 0.0;
  const int64_t full = n / r;
  const double f = (double)(n % r) / (double)r;
  const double part = f <= 0.0 ? 0.0 : (full == 0 ? 0.3 + 0.64 * f : 0.26 + 0.37 * f);
  return steps * ((double)full + part);
}

// Longest task (burn-in-step units per pair) of a core of core_len sites cut
// into K chunks with burn-in b, cut as chunk_cuts (windows.h) does with no
// window flanks: each interior boundary adds b forward steps to the right
// chunk and b backward steps to the left one, a core site costs w, and the
// cuts share the cost out evenly.
inline double chunk_steps(int64_t core_len, int K, int64_t b, double w) {
  if (K <= 1) return 2.0 * w * (double)core_len;
  return (2.0 * w * (double)core_len + 2.0 * (K - 1) * (double)b) / K;
}

// Size of the parts when n items are cut into as few parts of at most `cap`
// as possible, made as equal as possible: ceil(n / ceil(n / cap)).  Pair
// batches and pair chunks use it so no small last part runs on a mostly idle
// GPU (the per-site summary: 28,775 + 28,775 + 5,640 pairs took 0.265 s,
// three batches of 21,064 took 0.217 s).  With `multiple` > 1 the size is
// rounded up to a multiple of it, never above `cap` when `cap` is one.
inline int64_t even_part(int64_t n, int64_t cap, int64_t multiple = 1) {
  if (n <= 0 || cap <= 0) return std::max<int64_t>(1, cap);
  const int64_t part = cdiv(n, cdiv(n, cap));
  if (multiple <= 1) return part;
  return std::min<int64_t>(cap >= multiple ? cap : cdiv(cap, multiple) * multiple,
                           cdiv(part, multiple) * multiple);
}

// What the chunk count depends on besides the launch.
struct ChunkPolicy {
  int64_t burn_in = 2048;     // burn-in sites of a chunk
  int64_t max_chunk = 16384;  // longest chunk core once a window is cut (0: no cap)
};

// Chunks per window for a launch of `tasks` (window, pair tile) tasks on
// `resident_tiles` tiles.  When the tasks fill the GPU twice over, only as
// many as keep chunks within the cap: chunks of ~16k sites ran faster per
// step than whole 32k-site windows, by more than their burn-ins cost (the
// chromosome job, 32,768-site cores: whole 179.0 ms, two chunks 174.9,
// three 179-186, four 182.4).  Otherwise the K (chunks of at least two
// burn-ins, at most the cap long) that minimises launch_cost -- the burn-in
// steps each extra chunk adds against filling the last wave.  With a slot
// budget, a tile's forward-state slot holds ceil(core / K) rows of
// `row_bytes`, and only the tiles whose slots fit the budget run at once.
inline int choose_chunks(const ChunkPolicy& pol, int64_t tasks, int64_t resident_tiles,
                         int64_t core_len, double row_bytes = 0.0, double slot_budget = 0.0) {
  if (tasks <= 0 || resident_tiles <= 0 || core_len <= 0) return 1;
  const int64_t b = std::max<int64_t>(1, pol.burn_in);
  const int k_max = (int)std::max<int64_t>(1, std::min<int64_t>(1024, core_len / (2 * b)));
  // once a window is cut its chunks stay within the cap: with the same waves,
  // chunks of 15-17k sites ran faster than 33k-site ones (the per-site
  // summary's 23,600-pair batches over 400,000 sites: 0.25 s at 27 chunks,
  // 0.32 s at 12), as did the slice's 12.5k-site chunks
  const int k_min =
      pol.max_chunk > 0 ? (int)std::min<int64_t>(k_max, cdiv(core_len, pol.max_chunk)) : 1;
  if (tasks >= 2 * resident_tiles) return k_min;
  auto tiles_for = [&](int K) {
    if (slot_budget <= 0.0 || row_bytes <= 0.0) return resident_tiles;
    const double fit = slot_budget / ((double)cdiv(core_len, K) * row_bytes);
    return std::max<int64_t>(1, std::min<int64_t>(resident_tiles, (int64_t)fit));
  };
  // Near-ties go to the fewest chunks (fewest burn-ins and boundaries to
  // verify): within 1% of the cheapest.  (The slice: K = 4 at 1.002 of K = 9,
  // measured 31.7 ms against 33.0 at K = 8.  A wider 5% let 8,192 pairs x
  // 50,000 sites take K = 11 at 1.024 of K = 12: 7.45 ms against 6.86.)
  std::vector<double> cost(k_max + 1, 1e300);
  double lowest = 1e300;
  for (int K = k_min; K <= k_max; ++K) {
    cost[K] = launch_cost(tasks * K, tiles_for(K), chunk_steps(core_len, K, b, 1.0));
    lowest = std::min(lowest, cost[K]);
  }
  for (int K = k_min; K <= k_max; ++K)
    if (cost[K] <= 1.01 * lowest) return K;
  return k_min;
}

// A launch of several waves ends with the tasks that start last running on
// a partly empty GPU, where a lone task runs about three times faster than
// in a full wave but still for a whole chunk.  When the last wave is small
// (under a quarter of the resident tiles), the first window that can take
// it is cut in twice as many chunks, so the launch ends on half-length tasks
// (the chromosome job: 174.0 -> 169.8 and 176.1 -> 173.6 ms on two boxes;
// two windows, or one cut in four, gained less).  `K` holds the chunks of
// each window (every window has tiles_per_window tasks per chunk), `core`
// its core length; returns the window changed, or -1.
inline int split_tail(const ChunkPolicy& pol, int64_t tiles_per_window, int64_t resident_tiles,
                      const std::vector<int64_t>& core, std::vector<int>* K) {
  if (tiles_per_window <= 0 || resident_tiles <= 0 || K->size() != core.size()) return -1;
  // only launches whose whole windows fill the GPU twice over (the others
  // were planned by launch_cost, last wave included)
  if (tiles_per_window * (int64_t)K->size() < 2 * resident_tiles) return -1;
  int64_t n = 0;
  for (int k : *K) n += tiles_per_window * k;
  const int64_t last_wave = n % resident_tiles;
  if (last_wave == 0 || last_wave >= resident_tiles / 4) return -1;
  const int64_t b = std::max<int64_t>(1, pol.burn_in);
  for (size_t i = 0; i < K->size(); ++i) {
    if (2 * (int64_t)(*K)[i] <= core[i] / (2 * b)) {
      (*K)[i] *= 2;
      return (int)i;
    }
  }
  return -1;
}

}  // namespace plan
}  // namespace gsmc
