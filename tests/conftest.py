import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cb():
    import __graft_entry__ as ge
    return ge.load_package()


@pytest.fixture(scope="session")
def refh():
    import refh as r
    if not r.available():
        pytest.skip("reference harness oracle/_ref/libcfdref.so not built")
    return r


@pytest.fixture(scope="session")
def has_gpu(cb):
    return cb.device_count() > 0


def rel_err(a, b, axis_len=None):
    """max |a-b| / max |b| (per block of axis_len entries when given)."""
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if axis_len:
        a = a.reshape(-1, axis_len)
        b = b.reshape(-1, axis_len)
        scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
        return float((np.abs(a - b).max(axis=1) / scale).max())
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
