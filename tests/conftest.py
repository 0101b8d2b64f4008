import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "bem-cpp_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than ~20 s on the CPU")


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return {k: d[k] for k in d.files}


def golden_rwg(g):
    rwg = {k[4:]: g[k] for k in g if k.startswith("rwg_")}
    rwg["N"] = len(rwg["tri_p"])
    return rwg


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture
def golden():
    return load_golden
