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


def reference_dir():
    """The reference tree, where it is mounted: FKADJ_REFERENCE_DIR, else the
    directory oracle/ref_build.sh recorded when it built oracle/_ref; None
    when neither exists (a GPU box has no reference tree)."""
    d = os.environ.get("FKADJ_REFERENCE_DIR")
    if not d:
        rec = os.path.join(ROOT, "oracle", "_ref", "source_dir")
        if os.path.exists(rec):
            d = open(rec).read().strip()
    return d if d and os.path.isdir(d) else None


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
