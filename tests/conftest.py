import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine library")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def oracle_crpow():
    from oracle import Oracle
    return Oracle(cr_pow=True)


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library not built (make -C oracle ref needs the reference checkout)")
    return Reference()
