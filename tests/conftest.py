import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")
    config.addinivalue_line("markers", "slow: long-running")


def load_golden(name):
    """(domain, WINDSGeneralData, raw npz dict) for a golden case."""
    import qesb

    z = dict(np.load(os.path.join(GOLDEN, name)))
    d = qesb.Domain(int(z["Nx"]), int(z["Ny"]), int(z["Nz"]), float(z["dx"]), float(z["dy"]), 1.0,
                    z["dz_array"])
    w = qesb.WINDSGeneralData(d)
    for k in ("e", "f", "g", "h", "m", "n", "u0", "v0", "w0"):
        setattr(w, k, np.ascontiguousarray(z[k], np.float32))
    w.icellflag = np.ascontiguousarray(z["icellflag"], np.int32)
    return d, w, z


@pytest.fixture
def golden():
    return load_golden
