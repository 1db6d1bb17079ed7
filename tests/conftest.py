import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "senga-versiona_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def rel_linf(got, want):
    """Field-normalised relative L-infinity: max|got-want| / max|want|."""
    import numpy as np

    den = float(np.max(np.abs(want)))
    if den == 0.0:
        return float(np.max(np.abs(got)))
    return float(np.max(np.abs(got - want))) / den


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
