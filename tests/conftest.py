import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def rel_fro(a, b):
    import numpy as np
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.reshape(-1))
    return float(np.linalg.norm((a - b).reshape(-1)) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
