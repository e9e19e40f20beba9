import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

FLOW_FIELD = os.path.join(REPO, "gamma_smc_cu_b200", "data", "default_flow_field.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_built():
    """Build the product library and the oracle if they are missing (nvcc and
    g++ work without a GPU)."""
    from gamma_smc_cu_b200 import build as b
    if not os.path.exists(b.LIB):
        b.build()
    if not os.path.exists(os.path.join(REPO, "oracle", "_build", "libgsmc_oracle.so")):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle")], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def flow_field():
    return FLOW_FIELD


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O


@pytest.fixture(scope="session")
def small_data():
    from gamma_smc_cu_b200 import synthetic
    return synthetic.cohort("small")


@pytest.fixture(scope="session")
def ref_core():
    """The reference's own pybind11 module built from its sources for sm_100a
    into oracle/_ref (None when absent); loaded once per process."""
    import importlib.util
    from oracle import oracle as O
    path = O.ref_core_path()
    if path is None:
        return None
    spec = importlib.util.spec_from_file_location("_core", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod
