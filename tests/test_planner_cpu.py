"""The scan's launch planning on the CPU.

csrc/planner.h holds the arithmetic that decides how many exact speculative
chunks a window is cut into (the chunked decode is bit-identical to the
whole-window one, so only speed depends on it).  It is compiled here as plain
C++ and its decisions are pinned on the shapes they were measured on:

* the 50,000-site full-posterior slice, 63,190 pairs (247 two-pair tiles on
  1,184 resident tiles): 4 chunks (31.7 ms; 33.0 at 8, 41.7 at 5);
* the same window over 8,192 pairs (32 tiles): 12 chunks (6.86 ms; 7.45 at 11);
* the chromosome job (13 windows, 32,768-site cores, 247 tiles each): 2
  chunks per full window (174.9 ms against 179.0 whole) and one window cut
  in 4 because the last wave is small (169.8 against 174.0 ms);
* the per-site summary's per-pair means over 400,000 sites (batches of
  22,528 pairs, 176 one-pair tiles on 1,480): 25 chunks (0.27 s);
* pair batches cut evenly (63,190 pairs at most 28,775 per batch: three of
  21,064, not 28,775 + 28,775 + 5,640; 0.265 -> 0.217 s for the summary).
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "gamma_smc_cu_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "planner.h"
using namespace gsmc::plan;
int main() {
  char cmd[16];
  while (std::scanf("%15s", cmd) == 1) {
    long long burn, cap;
    std::scanf("%lld %lld", &burn, &cap);
    ChunkPolicy pol;
    pol.burn_in = burn;
    pol.max_chunk = cap;
    if (cmd[0] == 'e') {           // even part: n cap multiple (burn, cap read above unused)
      long long n, c, m;
      std::scanf("%lld %lld %lld", &n, &c, &m);
      std::printf("%lld\n", (long long)even_part(n, c, m));
    } else if (cmd[0] == 'c') {    // choose: tasks resident core row_bytes budget
      long long t, r, core;
      double rb, bud;
      std::scanf("%lld %lld %lld %lf %lf", &t, &r, &core, &rb, &bud);
      std::printf("%d\n", choose_chunks(pol, t, r, core, rb, bud));
    } else {                       // split: tiles resident n core... K...
      long long tiles, r;
      int n;
      std::scanf("%lld %lld %d", &tiles, &r, &n);
      std::vector<long long> c(n);
      std::vector<int64_t> core(n);
      std::vector<int> K(n);
      for (int i = 0; i < n; ++i) { std::scanf("%lld", &c[i]); core[i] = c[i]; }
      for (int i = 0; i < n; ++i) std::scanf("%d", &K[i]);
      const int w = split_tail(pol, tiles, r, core, &K);
      std::printf("%d", w);
      for (int k : K) std::printf(" %d", k);
      std::printf("\n");
    }
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("planner")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wno-unused-result", "-I", CSRC, str(src), "-o",
                    str(exe)], check=True)
    return str(exe)


def _run(driver, lines):
    out = subprocess.run([driver], input="".join(l + "\n" for l in lines), capture_output=True,
                         text=True, check=True).stdout.split("\n")
    return [o for o in out if o]


def choose(driver, tasks, resident, core, burn=2048, cap=16384, row_bytes=0.0, budget=0.0):
    return int(_run(driver, [f"c {burn} {cap} {tasks} {resident} {core} {row_bytes} {budget}"])[0])


def split(driver, tiles, resident, cores, K, burn=2048, cap=16384):
    line = f"s {burn} {cap} {tiles} {resident} {len(cores)} " + " ".join(map(str, cores)) + " " + \
        " ".join(map(str, K))
    v = [int(x) for x in _run(driver, [line])[0].split()]
    return v[0], v[1:]


def test_measured_shapes(driver):
    assert choose(driver, 247, 1184, 50_000) == 4          # slice, two pairs per thread
    assert choose(driver, 32, 1184, 50_000) == 12          # 8,192 pairs of the slice
    assert choose(driver, 176, 1480, 400_000) == 25        # summary batch, one pair per thread
    # chromosome job: 13 windows x 247 tiles fill the GPU twice -> the cap only
    assert choose(driver, 13 * 247, 1184, 32_768) == 2
    assert choose(driver, 13 * 247, 1184, 6_784) == 1     # the short last window
    cores = [32_768] * 12 + [6_784]
    w, K = split(driver, 247, 1184, cores, [2] * 12 + [1])
    assert w == 0 and K == [4] + [2] * 11 + [1]            # 6,175 tasks leave 255 in the last wave


def test_multiwave_test_shape(driver):
    # the shape tests/test_gpu_spec_multiwave.py runs: 16 windows of 512-site
    # cores, burn-in 64, cap 256 -> two chunks each, last wave 800 of 1,184
    assert choose(driver, 16 * 247, 1184, 512, burn=64, cap=256) == 2
    w, K = split(driver, 247, 1184, [512] * 16, [2] * 16, burn=64, cap=256)
    assert w == -1 and K == [2] * 16


def test_edges(driver):
    assert choose(driver, 0, 1184, 50_000) == 1
    assert choose(driver, 10, 1184, 3_000) == 1            # shorter than two burn-ins
    assert choose(driver, 10, 1184, 50_000, cap=0) >= 1
    # no cap: a window that fills the GPU twice is not cut
    assert choose(driver, 13 * 247, 1184, 32_768, cap=0) == 1
    # a full last wave, or launches planned by the cost model, are left alone
    w, K = split(driver, 296, 1184, [32_768] * 8, [2] * 8)
    assert w == -1
    w, K = split(driver, 247, 1184, [50_000], [4])
    assert w == -1 and K == [4]
    # windows already at their most chunks (two burn-ins each) are skipped
    w, K = split(driver, 247, 1184, [8_192] * 13, [2] * 12 + [1])
    assert w == 12 and K == [2] * 13


def test_slot_budget_prefers_shorter_chunks(driver):
    # one tile's slot: core / K rows of 2 KB; with room for only 200 whole-
    # window slots the plan cuts the window so more tiles can run
    whole = choose(driver, 247, 1184, 50_000)
    tight = choose(driver, 247, 1184, 50_000, row_bytes=2048.0, budget=200 * 50_000 * 2048.0)
    assert tight >= whole


def even(driver, n, cap, multiple=1):
    return int(_run(driver, [f"e 0 0 {n} {cap} {multiple}"])[0])


def test_even_parts(driver):
    # the summary's pair batches: 63,190 pairs, at most 28,775 per batch
    assert even(driver, 63_190, 28_775) == 21_064
    assert even(driver, 63_190, 25_002) == 21_064
    assert even(driver, 63_190, 63_190) == 63_190
    assert even(driver, 63_190, 100_000) == 63_190
    assert even(driver, 600, 250) == 200                  # three batches of 200
    for n in (1, 7, 255, 256, 257, 1000, 63_190, 1_000_000):
        for cap in (1, 3, 100, 256, 1000, 31_595, 2_000_000):
            p = even(driver, n, cap)
            k = -(-n // cap)
            assert p <= cap and -(-n // p) == k           # same number of parts, none over cap
            assert p * k - n < k                          # parts differ by at most one
            q = even(driver, n, max(cap, 256) // 256 * 256, 256)
            assert q % 256 == 0 and q <= max(cap, 256) // 256 * 256
            assert -(-n // q) == -(-n // (max(cap, 256) // 256 * 256))
