import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "softx-d-21-00092_b200")
for p in (os.path.join(REPO, "tests"), PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from jwref import Oracle
    return Oracle()


def golden(name):
    import numpy as np
    return dict(np.load(os.path.join(REPO, "tests", "golden", f"{name}.npz"), allow_pickle=False))


@pytest.fixture(scope="session")
def gold():
    return golden
