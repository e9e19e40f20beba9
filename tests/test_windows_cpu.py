"""Window arithmetic of the blockwise decoders, on the CPU.

csrc/windows.h holds the one definition of the blockwise windows (core
[cs, ce) padded by flank sites on both sides, clamped to the sequence;
src/bindings.cpp:2517-2534 in the reference) that the context planner and the
allocation-free kernel share.  Here it is compiled as plain C++ and compared,
for extreme int64 core and flank values, against the same definition in
unbounded Python integers: every bound must lie in [0, n_sites], so no kernel
can index outside the sequence whatever the caller passes.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "gamma_smc_cu_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "windows.h"
int main() {
  long long S, core, flank;
  while (std::scanf("%lld %lld %lld", &S, &core, &flank) == 3) {
    const long long n = gsmc::window_count(S, core);
    std::printf("%lld", n);
    const long long ws[3] = {0, n / 2, n - 1};
    for (long long w : ws) {
      if (n == 0) break;
      const gsmc::WindowBounds b = gsmc::window_bounds(w, S, core, flank);
      std::printf(" %lld %lld %lld %lld %lld", w, (long long)b.ps, (long long)b.cs,
                  (long long)b.ce, (long long)b.pe);
    }
    std::printf("\n");
  }
  return 0;
}
"""

INT64_MAX = 2**63 - 1


def _expected(S, core, flank, w):
    cs = w * core
    ce = min(S, cs + core)
    return max(0, cs - flank), cs, ce, min(S, ce + flank)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("windows")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return str(exe)


def test_window_bounds_stay_in_the_sequence(driver):
    sizes = [1, 2, 7, 1000, 400_000, 2**31 - 2]
    cores = [1, 3, 1024, 32_768, 2**31 - 1, 2**40, INT64_MAX]
    flanks = [0, 1, 2048, 2**31 - 1, 2**31, 2**40, INT64_MAX]
    cases = [(S, c, f) for S in sizes for c in cores for f in flanks
             if (S + c - 1) // c <= 10**9]  # keep the window counts printable
    inp = "".join(f"{S} {c} {f}\n" for S, c, f in cases)
    out = subprocess.run([driver], input=inp, capture_output=True, text=True, check=True).stdout
    lines = out.strip().splitlines()
    assert len(lines) == len(cases)
    for (S, core, flank), line in zip(cases, lines):
        v = [int(x) for x in line.split()]
        n = (S + core - 1) // core
        assert v[0] == n, (S, core, flank)
        for k in range(1, len(v), 5):
            w, ps, cs, ce, pe = v[k:k + 5]
            assert (ps, cs, ce, pe) == _expected(S, core, flank, w), (S, core, flank, w)
            assert 0 <= ps <= cs < ce <= pe <= S, (S, core, flank, w)


def test_zero_sites_has_no_window(driver):
    out = subprocess.run([driver], input="0 5 3\n", capture_output=True, text=True,
                         check=True).stdout
    assert out.strip() == "0"


CUTS_DRIVER = r"""
#include <cstdio>
#include "windows.h"
int main() {
  long long ps, cs, ce, pe, flank;
  int K;
  double w;
  while (std::scanf("%lld %lld %lld %lld %d %lld %lf", &ps, &cs, &ce, &pe, &K, &flank, &w) == 7) {
    long long cut[1100];
    int64_t c64[1100];
    gsmc::chunk_cuts(ps, cs, ce, pe, K, flank, w, c64);
    for (int k = 0; k <= K; ++k) cut[k] = c64[k];
    for (int k = 0; k <= K; ++k) std::printf("%lld ", cut[k]);
    std::printf("\n");
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def cuts_driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("cuts")
    src = d / "cuts.cpp"
    src.write_text(CUTS_DRIVER)
    exe = d / "cuts"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return str(exe)


def _steps(ps, cs, ce, pe, flank, cut, w=1.0):
    K = len(cut) - 1
    out = []
    for k in range(K):
        pre = cs - ps if k == 0 else flank
        post = pe - ce if k == K - 1 else flank
        out.append(2 * w * (cut[k + 1] - cut[k]) + pre + post)
    return out


def test_chunk_cuts_balance_pair_steps(cuts_driver):
    """Speculative chunk cuts cover the core exactly, in order, and give every
    chunk the same forward + backward steps (to rounding): a chunk at a
    sequence end, which runs no burn-in on that side, gets the steps as
    extra core.  Windows with flanks on both sides as long as the burn-in
    are cut into equal lengths."""
    cases = [
        (0, 0, 50_000, 50_000, 4, 2048),           # one window over a whole slice
        (0, 0, 50_000, 50_000, 9, 2048),
        (0, 0, 32_768, 34_816, 3, 2048),            # first window of a chromosome
        (30_720, 32_768, 65_536, 67_584, 5, 2048),  # interior window
        (393_216 - 2048, 393_216, 400_000, 400_000, 2, 2048),
        (0, 0, 400_000, 400_000, 25, 2048),
        (0, 0, 10, 10, 3, 2048),                    # too short: equal lengths
        (0, 0, 1 << 40, 1 << 40, 1000, 2048),
    ]
    cases += [case[:6] + (1.5,) for case in cases[:6]]
    cases = [c if len(c) == 7 else c + (1.0,) for c in cases]
    inp = "".join(f"{a} {b} {c} {d} {K} {f} {w}\n" for a, b, c, d, K, f, w in cases)
    out = subprocess.run([cuts_driver], input=inp, capture_output=True, text=True,
                         check=True).stdout.strip().splitlines()
    assert len(out) == len(cases)
    for (ps, cs, ce, pe, K, flank, w), line in zip(cases, out):
        cut = [int(x) for x in line.split()]
        assert len(cut) == K + 1
        assert cut[0] == cs and cut[-1] == ce
        assert all(b > a for a, b in zip(cut, cut[1:])) or ce - cs < K
        lens = [b - a for a, b in zip(cut, cut[1:])]
        if min(lens) < flank:
            # fallback: the equal-length cuts
            assert cut == [cs + (ce - cs) * k // K for k in range(K + 1)]
            continue
        st = _steps(ps, cs, ce, pe, flank, cut, w)
        assert max(st) - min(st) <= 4 * w, (ps, cs, ce, pe, K, w, st)
        if cs - ps == flank and pe - ce == flank:
            assert max(lens) - min(lens) <= 2
    # the slice: an edge chunk runs one burn-in fewer and takes its cost as
    # core, flank / (2 w) sites more (a core site is walked forward and
    # backward, w burn-in sites each): 1,024 at w = 1, 683 at w = 1.5
    cut = [int(x) for x in out[0].split()]
    assert [b - a for a, b in zip(cut, cut[1:])] == [13012, 11988, 11988, 13012]
    cut = [int(x) for x in out[8].split()]
    lens = [b - a for a, b in zip(cut, cut[1:])]
    assert lens[0] == lens[3] and lens[1] == lens[2] and abs(lens[0] - lens[1] - 683) <= 2
