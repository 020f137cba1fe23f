import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "fixtures.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port

    return Port()


@pytest.fixture(scope="session")
def reference():
    """The reference's own bfs.hpp (oracle/_ref), or None where it was never built."""
    from oracle import oracle as O

    try:
        return O.Reference()
    except (FileNotFoundError, OSError):
        return None


class GoldenGraph:
    def __init__(self, z, name):
        self.name = name
        self.off = z[f"{name}/off"]
        self.cols = z[f"{name}/cols"]
        self.in_off = z[f"{name}/in_off"] if f"{name}/in_off" in z else None
        self.in_cols = z[f"{name}/in_cols"] if f"{name}/in_cols" in z else None
        self.roots = z[f"{name}/roots"]
        self.depths = z[f"{name}/depths"]
        self.ref_ok = z[f"{name}/ref_verifier_ok"]
        self.trace_dir = [z[f"{name}/trace_dir/{i}"] for i in range(self.roots.size)]
        self.trace_found = [z[f"{name}/trace_found/{i}"] for i in range(self.roots.size)]

    @property
    def n(self):
        return self.off.size - 1


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN)
    return [GoldenGraph(z, str(nm)) for nm in z["names"]]


@pytest.fixture(scope="session")
def nwg():
    """The CUDA library; built in-tree first if it is missing (nvcc only)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("nwgr_b200_build", os.path.join(ROOT, "nwgr_b200", "build.py"))
    B = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(B)
    B.build()
    import nwgr_b200

    return nwgr_b200
