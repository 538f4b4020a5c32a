import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs libkls.so kernels)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


def load_case(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def lib_path():
    from kalnajs_log_spirals_b200 import build
    return build.build()
