import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_cases(prefix):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle.orc import Oracle
    return Oracle()


def rel_fro(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def same_oidx(keys_of, oidx_a, oidx_b):
    """oidx rows agree as groupings: identical mode-index sequence and, for
    each index value, the same set of nonzero positions (tie order is the
    sort's choice in the reference)."""
    ka, kb = keys_of(oidx_a), keys_of(oidx_b)
    if not np.array_equal(ka, kb):
        return False
    order_a = np.lexsort((oidx_a, ka))
    order_b = np.lexsort((oidx_b, kb))
    return np.array_equal(oidx_a[order_a], oidx_b[order_b])
