import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "ka_*.npz")))


def load_golden(path):
    d = np.load(path)
    out = {k: d[k] for k in d.files}
    out["name"] = os.path.basename(path)[3:-4]
    return out


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O
