import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle_ffi
    oracle_ffi.lib()
    return oracle_ffi


@pytest.fixture
def ctx_factory():
    """Builds rbmd_b200 contexts; the library must be present (no CPU path)."""
    import rbmd_b200
    made = []

    def make(**kw):
        c = rbmd_b200.Context(**kw)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.sqrt((b * b).sum())
    return float(np.sqrt(((a - b) ** 2).sum()) / (den if den > 0 else 1.0))
