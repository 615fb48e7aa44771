import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mst-artifact-sc23_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size inputs (minutes on the CPU oracle)")


@pytest.fixture(scope="session")
def golden():
    data = np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))
    cases = {}
    for name in data["names"]:
        name = str(name)
        cases[name] = {k: data[f"{name}/{k}"] for k in ("nindex", "nlist", "eweight", "inMST", "threshold")}
    return cases
