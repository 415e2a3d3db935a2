import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdense_b200.so")


def gpu_available() -> bool:
    try:
        from opensfm_b200 import _lib
        return _lib.load().dn_device_count() > 0
    except OSError:
        return False


@pytest.fixture(scope="session")
def golden():
    d = os.path.join(ROOT, "tests", "golden")

    def load(name):
        return dict(np.load(os.path.join(d, name)))
    return load


def cams(vs):
    return ([c.K for c in vs.cameras], [c.R for c in vs.cameras], [c.t for c in vs.cameras])
