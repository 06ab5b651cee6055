import importlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

PKG_NAME = "gpu-canonical-labeling_b200"

# Bound every graph's device search in tests: a regression that loops stops
# with GCL_ERR_TIMEOUT instead of holding the GPU.
os.environ.setdefault("GCL_GRAPH_BUDGET_S", "30")
# one hardware work queue per stream for the serving tests' many lanes
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "gpu_staged: needs a B200; not yet run on one "
                                       "(pytest -m gpu_staged)")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module(PKG_NAME)


@pytest.fixture(scope="session")
def G():
    return importlib.import_module(PKG_NAME + ".graphs")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)["records"]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle  # noqa: F401  (oracle/oracle.py, test infrastructure)
    if not oracle.available("port"):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return oracle


def golden_graph(G, rec):
    import numpy as np
    e = np.asarray(rec["edges"], dtype=np.int64).reshape(-1, 2)
    return G.from_edges(rec["n"], e, rec["color"])
