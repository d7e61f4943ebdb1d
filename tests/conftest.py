import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    n = len(z["indptr"]) - 1
    return sp.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
