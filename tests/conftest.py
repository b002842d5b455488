import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def ref():
    """The reference sources compiled through the stand-in headers."""
    from oracle.oracle import reference
    o = reference()
    if o is None:
        pytest.skip("oracle/_ref/libaxref.so not built (reference checkout absent)")
    return o


@pytest.fixture(scope="session")
def engine():
    from asterx_b200.engine import Engine
    e = Engine(0)
    yield e
    e.close()
