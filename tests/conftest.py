import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def ref_small():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "ref_small.npz")))


@pytest.fixture(scope="session")
def sod_check():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "sod_check.json")) as f:
        return json.load(f)
