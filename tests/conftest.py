"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def grlbm():
    return importlib.import_module("2dradiation_b200")


@pytest.fixture(scope="session")
def W(grlbm):
    return grlbm.workloads


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    if not O.available("oracle"):
        O.build(with_reference=False)
    return O


def rel_l2(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))

GOLDEN = Path(__file__).resolve().parent / "golden"
if str(GOLDEN) not in sys.path:
    sys.path.insert(0, str(GOLDEN))


@pytest.fixture(scope="session")
def cases(W):
    from cases import golden_cases
    return golden_cases(W)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = dict(np.load(GOLDEN / f"{name}.npz"))
        return cache[name]
    return load


GOLDEN_NAMES = ["flat_beam", "curved_shell", "curved_scatter", "moving_kerr", "moving_schwarzschild",
                "moving_flat", "shipped_constants"]
