import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def relerr(a, b):
    """max |a-b| / max |b| (0 if both are zero)."""
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if b.size else 0.0
    if den == 0.0:
        return num
    return num / den


@pytest.fixture(scope="session")
def has_gpu():
    from ixchel2d_b200 import lib
    return lib.ixb_device_count() > 0
