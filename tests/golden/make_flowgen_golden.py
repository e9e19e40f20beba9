"""Golden flow fields from the reference's own generator, for the GPU generator.

Imports ``generate_flow_field`` from a reference checkout
(``python/gamma_smc_cu/demographic.py:146-208``; numpy/scipy only, with a stub
``_core``) and stores its raw float64 output -- not rounded, not sanitised --
for a constant-Ne grid and a three-epoch demographic grid.

    python tests/golden/make_flowgen_golden.py [/path/to/reference]

Writes ``tests/golden/flowgen.npz``.
"""
from __future__ import annotations

import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_flow_field import _load_reference_demographic  # noqa: E402

CASES = {
    "const": {},
    "demo": {"Ne_values": [2.0e4, 5.0e3, 1.5e4], "epoch_boundaries": [0.0, 2.0e3, 3.0e4],
             "Ne_ref": 1.0e4, "n_steps": 200},
}


def main(ref_root: str = "/root/reference") -> None:
    demo = _load_reference_demographic(ref_root)
    out = {}
    for name, kw in CASES.items():
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            u, v = demo.generate_flow_field(verbose=False, **kw)
        out[f"{name}_u"] = u
        out[f"{name}_v"] = v
    path = os.path.join(HERE, "flowgen.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}")


if __name__ == "__main__":
    main(*sys.argv[1:])
