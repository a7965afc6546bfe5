import os
import sys

# one BLAS thread per process: the oracle's dense eigen-solves run fastest
# single-threaded here, and parallel test processes must not oversubscribe
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("OMP_NUM_THREADS", "1")

import pytest  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes tens of seconds on CPU")


def golden_path(name):
    return os.path.join(ROOT, "tests", "golden", name)


@pytest.fixture(scope="session")
def dev500():
    import numpy as np
    return np.load(golden_path("dev500x50.npz"))


@pytest.fixture(scope="session")
def dev500_trace():
    import json
    with open(golden_path("dev500x50_trace.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def lib_built():
    """Build the CUDA library in-tree if it is missing (nvcc cross-compiles)."""
    import fastkpc_b200
    from fastkpc_b200 import build
    if not os.path.exists(fastkpc_b200.library_path()):
        build.build()
    return fastkpc_b200.load_library()
