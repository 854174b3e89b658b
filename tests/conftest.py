import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libg2s_b200.so")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def oracle():
    from oracle import qs_oracle
    if not qs_oracle.available():
        pytest.fail("oracle/_ref/libqsoracle.so is missing: run `make -C oracle oracle`")
    return qs_oracle


@pytest.fixture(scope="session")
def g2s():
    import g2s_b200
    return g2s_b200


@pytest.fixture(scope="session")
def gpu(g2s):
    n = g2s.device_count()
    if n < 1:
        pytest.fail("no CUDA device visible to libg2s_b200.so")
    return 0
