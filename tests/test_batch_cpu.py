"""Host logic of batched jobs (no GPU): batch layout, task counts, and the
ctypes structures against the C header's layout."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from gamma_smc_cu_b200 import _lib
from gamma_smc_cu_b200.batch import Job, Layout, _count_tasks, validate

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_job_normalises_pairs():
    j = Job([(3, 1), (2, 0)], 5, 9, mean_only=False, return_posterior=True)
    assert j.pairs.dtype == np.int32 and j.pairs.shape == (2, 2)
    assert (j.rows, j.n_pairs, j.n_outputs, j.pair_sites) == (4, 2, 5, 8)
    assert j.flags == _lib.GSMC_CI | _lib.GSMC_POSTERIOR
    assert Job([], 0, 3).n_pairs == 0
    with pytest.raises(TypeError):
        Job([1, 2, 3], 0, 3)


def test_validate():
    validate(Job([(3, 1)], 0, 10), 4, 10)
    with pytest.raises(ValueError, match="out of range"):
        validate(Job([(3, 1)], 0, 11), 4, 10)
    with pytest.raises(ValueError, match="out of range"):
        validate(Job([(3, 1)], 6, 5), 4, 10)
    with pytest.raises(ValueError, match="pair index"):
        validate(Job([(4, 1)], 0, 10), 4, 10)
    with pytest.raises(ValueError, match="pair index"):
        validate(Job([(-1, 1)], 0, 10), 4, 10)


def test_layout_packs_pairs_and_outputs():
    jobs = [Job([(1, 0), (2, 0), (2, 1)], 0, 5), Job([(3, 2)], 2, 4, mean_only=False),
            Job(np.zeros((0, 2)), 0, 7, return_posterior=True)]
    lay = Layout(jobs)
    pairs = np.full(lay.pair_ints, -1, np.int32)
    lay.pack_pairs(pairs)
    assert pairs.tolist() == [1, 2, 2, 0, 0, 1, 3, 2]
    # outputs: job 0 mean (15 -> 64 floats), job 1 mean/lower/upper (2 each -> 64 each)
    assert lay.out_off[0].tolist() == [0, -1, -1, -1, -1]
    assert lay.out_off[1].tolist() == [64, 128, 192, -1, -1]
    assert lay.out_off[2].tolist() == [256, -1, -1, 256, 256]
    assert [r[:2] for r in lay.regions()] == [(0, "mean"), (1, "mean"), (1, "lower"),
                                              (1, "upper")]
    arr = lay.c_jobs(1000, 50000)
    assert arr[1].pair_i == 1000 + 4 * 6 and arr[1].pair_j == 1000 + 4 * 7
    assert arr[1].out[0] == 50000 + 4 * 64 and arr[1].out[3] is None
    assert (arr[1].site_begin, arr[1].site_end, arr[1].ld_out, arr[1].flags) == (2, 4, 1, 1)
    host = np.arange(lay.out_floats, dtype=np.float32)
    res = lay.results(host)
    assert res[0]["mean"].shape == (5, 3) and res[0]["mean"][1, 0] == 3
    assert set(res[1]) == {"mean", "lower", "upper"} and res[1]["lower"][0, 0] == 128
    assert res[2]["posterior_alpha"].shape == (7, 0)


def test_count_tasks_bounds_executor_tasks():
    jobs = [Job(np.zeros((70, 2)), 0, 10000), Job(np.zeros((1, 2)), 0, 10)]
    assert _count_tasks(jobs, {}) == 3 + 1
    assert _count_tasks(jobs, {"core_block_sites": 4096}) == 3 * 3 + 1
    assert _count_tasks(jobs, {"tile_width": 128, "pairs_per_thread": 2}) == 2


def test_ctypes_structs_match_header(tmp_path):
    """Compile a probe against include/gsmc_b200.h and compare sizes/offsets."""
    src = tmp_path / "probe.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "gsmc_b200.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m))
int main(void) {
  printf("gsmc_job %zu\n", sizeof(gsmc_job));
  printf("gsmc_exec_config %zu\n", sizeof(gsmc_exec_config));
  F(gsmc_job, n_pairs); F(gsmc_job, site_end); F(gsmc_job, flags); F(gsmc_job, out);
  F(gsmc_job, ld_out); F(gsmc_job, out_col0);
  F(gsmc_exec_config, core_block_sites); F(gsmc_exec_config, max_pool_bytes);
  F(gsmc_exec_config, max_ctas); F(gsmc_exec_config, use_graph);
  return 0;
}
''')
    exe = tmp_path / "probe"
    r = subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode:
        pytest.skip("no C compiler: " + r.stderr[:200])
    got = dict(l.rsplit(" ", 1) for l in subprocess.check_output([str(exe)], text=True).split("\n") if l)
    assert int(got["gsmc_job"]) == ctypes.sizeof(_lib.Job)
    assert int(got["gsmc_exec_config"]) == ctypes.sizeof(_lib.ExecConfig)
    for name, val in got.items():
        if "." in name:
            T, m = name.split(".")
            cls = _lib.Job if T == "gsmc_job" else _lib.ExecConfig
            assert getattr(cls, m).offset == int(val), name


def test_job_mix_bp_windows_cover_their_sequence():
    from gamma_smc_cu_b200 import synthetic
    G, pos = synthetic.cohort("small")
    jobs = synthetic.job_mix_bp(pos, G.shape[0], 512, seed=5)
    assert len(jobs) == 512
    S = G.shape[1]
    for j in jobs:
        assert 0 <= j["site_begin"] < j["site_end"] <= S
        assert 1 <= len(j["pairs"]) <= G.shape[0] * (G.shape[0] - 1) // 2
        assert len({tuple(p) for p in j["pairs"]}) == len(j["pairs"])
    widths = [j["site_end"] - j["site_begin"] for j in jobs]
    assert max(widths) < S and min(widths) >= 1   # 200 kb of a 1 Mb sequence at most
    assert synthetic.job_mix_bp(pos, G.shape[0], 512, seed=5)[7]["site_begin"] == jobs[7]["site_begin"]


def test_layout_floats_match_job_padding():
    """The server admits queries by Job.layout_floats; a batch's buffer is the
    sum of those (every output region padded to the layout's alignment)."""
    from gamma_smc_cu_b200.batch import Job, Layout
    rng = np.random.default_rng(3)
    jobs = []
    for k in range(40):
        n = int(rng.integers(1, 70))
        s0 = int(rng.integers(0, 400))
        jobs.append(Job(np.stack([rng.integers(1, 20, n), np.zeros(n, int)], 1), s0,
                        s0 + int(rng.integers(1, 300)), mean_only=k % 3 != 0,
                        return_posterior=k % 4 == 1))
    lay = Layout(jobs)
    assert lay.out_floats == sum(j.layout_floats for j in jobs)
    assert all(j.layout_floats >= j.output_floats for j in jobs)
