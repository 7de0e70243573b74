import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def relerr(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    import numpy as np
    den = float(np.abs(b).max())
    num = float(np.abs(a - b).max())
    return num / den if den > 0 else num
