"""Generate the flow-field fixture shared by the oracle, the tests and the product.

The reference loads its flow field from upstream gamma_smc's
``default_flow_field.txt`` (``src/flow_field.cpp:8-54``), a resource file that
is not shipped with the reference.  The reference does ship a generator for
the same 51 x 50 grid, ``generate_flow_field`` in
``python/gamma_smc_cu/demographic.py:146-208`` (constant-Ne path), and a
writer, ``write_flow_field`` (``demographic.py:215-220``).  This script imports
those two functions from a reference checkout (with a stub ``_core`` module,
since only numpy/scipy code runs) and writes the result.

Sanitisation: the generator leaves non-finite or huge values (|x| > 1e3) in
rows 0-8, the corner of the grid with log10(mean) <= -3.74 and tiny CV, next
to the cells that the generator itself skips and leaves at exactly 0.  Those
cells are set to 0 as well, the generator's own value for cells it cannot fit.

Parity is defined on this file: the oracle and the CUDA path read the same
bytes.  Usage::

    python tests/golden/make_flow_field.py [/path/to/reference]

Writes ``gamma_smc_cu_b200/data/default_flow_field.txt`` and
``tests/golden/flow_field.sha256``.
"""
from __future__ import annotations

import hashlib
import importlib.util
import os
import sys
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(REPO, "gamma_smc_cu_b200", "data", "default_flow_field.txt")
SHA = os.path.join(HERE, "flow_field.sha256")


def _load_reference_demographic(ref_root: str):
    pkg = types.ModuleType("gamma_smc_cu")
    pkg.__path__ = []
    core = types.ModuleType("gamma_smc_cu._core")
    pkg._core = core
    sys.modules.setdefault("gamma_smc_cu", pkg)
    sys.modules.setdefault("gamma_smc_cu._core", core)
    path = os.path.join(ref_root, "python", "gamma_smc_cu", "demographic.py")
    spec = importlib.util.spec_from_file_location("gamma_smc_cu.demographic", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(ref_root: str = "/root/reference") -> None:
    demo = _load_reference_demographic(ref_root)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        u, v = demo.generate_flow_field(verbose=False)
    bad = ~np.isfinite(u) | ~np.isfinite(v) | (np.abs(u) > 1e3) | (np.abs(v) > 1e3)
    u = np.where(bad, 0.0, u)
    v = np.where(bad, 0.0, v)
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    demo.write_flow_field(OUT, u, v)
    digest = hashlib.sha256(open(OUT, "rb").read()).hexdigest()
    with open(SHA, "w") as f:
        f.write(f"{digest}  default_flow_field.txt\n")
    print(f"wrote {OUT} ({int(bad.sum())} cells sanitised) sha256={digest}")


if __name__ == "__main__":
    main(*sys.argv[1:])
