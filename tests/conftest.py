import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "adjoint-optimization_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "ref256.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA) and the built libfkadj")
    config.addinivalue_line("markers", "slow: long CPU oracle run (seconds to a minute)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
