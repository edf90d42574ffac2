import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libwmles_cuda.so")


def api_namespace():
    """This package's public classes under the names the case builders expect."""
    import wmles_jax_b200 as wm
    return types.SimpleNamespace(**{k: getattr(wm, k) for k in wm.__all__ if k != "Solver"})


@pytest.fixture(scope="session")
def W():
    return api_namespace()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "golden_cases.npz")))


@pytest.fixture(scope="session")
def golden_cfg1():
    return dict(np.load(os.path.join(GOLDEN, "golden_channel_cfg1.npz")))
