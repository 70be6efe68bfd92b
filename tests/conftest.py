"""Shared test set-up.

Marker ``gpu``: needs a B200; everything else runs on the CPU.  The oracle
(oracle/) is the checker; the product is libplategpu.so through its C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "gpu-gauntlet_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def gpu_ctx():
    from plategpu import _lib
    ctx = _lib.Context(0)
    yield ctx
    ctx.close()


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def max_w(x):
    """Signed w of largest magnitude (benchmark/page.tsx:121-127)."""
    w = np.asarray(x, np.float64)[0::3]
    return float(w[np.argmax(np.abs(w))])
