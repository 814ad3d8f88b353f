import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import pyoracle
    if not os.path.exists(pyoracle.REF_SO):
        pytest.skip("reference CPU library not built (oracle/_ref)")
    return pyoracle.RefLib()


@pytest.fixture(scope="session")
def ctx():
    from menos_b200 import Context
    return Context(0)
