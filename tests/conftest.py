import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def cp():
    import circlepacking_b200 as cp

    cp.lib()
    return cp


@pytest.fixture(scope="session")
def ref():
    from oracle import refcheck

    if not refcheck.available():
        pytest.fail(f"reference checker {refcheck.SO} is missing (build: make -C oracle ref)")
    refcheck.lib()
    return refcheck
