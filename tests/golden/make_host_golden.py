"""Golden vectors for the host-side logic of the path, made by the reference.

Imports the reference's own ``python/gamma_smc_cu/infer.py`` (with a stub
``_core``; only numpy code runs) and records its outputs on seeded inputs:

* ``_estimate_scaled_params``   (infer.py:44-99), incl. the known answers of
  tests/unit/test_infer.py:98-144 and the fallback cases;
* ``_filter_segregating``       (infer.py:102-126);
* ``_gpu_bytes_per_pair_site``, ``_estimate_block_gpu_bytes``,
  ``_recommend_core_block_size`` (infer.py:151-214).

Writes ``tests/golden/host_logic.json``.  Usage::

    python tests/golden/make_host_golden.py [/path/to/reference]
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "host_logic.json")


def load_reference_infer(ref_root):
    pkg = types.ModuleType("gamma_smc_cu")
    pkg.__path__ = []
    core = types.ModuleType("gamma_smc_cu._core")
    pkg._core = core
    sys.modules.setdefault("gamma_smc_cu", pkg)
    sys.modules.setdefault("gamma_smc_cu._core", core)
    path = os.path.join(ref_root, "python", "gamma_smc_cu", "infer.py")
    spec = importlib.util.spec_from_file_location("gamma_smc_cu.infer", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref_root="/root/reference"):
    ref = load_reference_infer(ref_root)
    rng = np.random.default_rng(20261203)
    theta = []
    # known answers from the reference's unit tests
    theta.append(dict(G=[[0, 0, 1, 1], [0, 1, 1, 1], [0, 0, 0, 1], [1, 0, 0, 1]],
                      positions=[10.0, 20.0, 30.0, 40.0], mu=2e-8, rho=5e-8, Ne=10000.0))
    theta.append(dict(G=[[0, 1], [1, 1], [0, 0], [0, 1]], positions=[100.0, 200.0],
                      mu=2e-8, rho=5e-8, Ne=10000.0))
    # fallbacks: odd n, n < 2, no sites, no hets
    theta.append(dict(G=[[0, 1, 1], [1, 0, 1], [1, 1, 0]], positions=[5.0, 9.0, 30.0],
                      mu=1.25e-8, rho=1e-8, Ne=10000.0))
    theta.append(dict(G=[[0, 1, 1]], positions=[5.0, 9.0, 30.0], mu=1.25e-8, rho=1e-8, Ne=1e4))
    theta.append(dict(G=[[], []], positions=[], mu=1.25e-8, rho=1e-8, Ne=1e4))
    theta.append(dict(G=[[0, 1], [0, 1]], positions=[3.0, 8.0], mu=1.25e-8, rho=1e-8, Ne=1e4))
    for k in range(8):
        n = int(rng.integers(1, 12)) * 2
        S = int(rng.integers(1, 200))
        G = (rng.random((n, S)) < rng.uniform(0.05, 0.6)).astype(np.uint8)
        pos = np.cumsum(rng.integers(1, 500, S)).astype(np.float64)
        theta.append(dict(G=G.tolist(), positions=pos.tolist(), mu=float(rng.uniform(5e-9, 3e-8)),
                          rho=float(rng.uniform(1e-9, 3e-8)), Ne=float(rng.integers(1000, 50000))))
    for case in theta:
        G = np.array(case["G"], dtype=np.uint8).reshape(len(case["G"]), -1)
        pos = np.array(case["positions"], dtype=np.float64)
        case["expected"] = list(ref._estimate_scaled_params(G, pos, case["mu"], case["rho"], case["Ne"]))

    seg = []
    for k in range(6):
        n = int(rng.integers(2, 10))
        S = int(rng.integers(1, 80))
        G = (rng.random((n, S)) < rng.uniform(0.0, 1.0)).astype(np.uint8)
        G[:, rng.random(S) < 0.2] = 0
        G[:, rng.random(S) < 0.2] = 1
        pos = np.arange(S, dtype=np.float64) * 10.0
        _, _, keep = ref._filter_segregating(G, pos)
        seg.append(dict(G=G.tolist(), keep=keep.astype(int).tolist()))

    sizing = []
    for n_sites in (217, 5000, 400_000):
        for n_pairs in (0, 1, 2, 780, 63_190, 1_000_000):
            for mean_only in (True, False):
                for flank in (0, 64, 2048):
                    for free in (1024, 512 * 2**20, 3 * 10**9, 32 * 10**9, 178 * 10**9):
                        core, est = ref._recommend_core_block_size(n_sites, n_pairs, mean_only,
                                                                   flank, free)
                        sizing.append(dict(n_sites=n_sites, n_pairs=n_pairs, mean_only=mean_only,
                                           flank=flank, free=free, core=int(core), est=int(est),
                                           est_clamped=int(ref._estimate_block_gpu_bytes(
                                               8192, flank, n_pairs, mean_only, n_sites=n_sites))))
    bps = {str(m): ref._gpu_bytes_per_pair_site(m) for m in (True, False)}
    with open(OUT, "w") as f:
        json.dump(dict(theta=theta, segregating=seg, sizing=sizing, bytes_per_pair_site=bps), f)
    print(f"wrote {OUT}: {len(theta)} theta, {len(seg)} filter, {len(sizing)} sizing cases")


if __name__ == "__main__":
    main(*sys.argv[1:])
