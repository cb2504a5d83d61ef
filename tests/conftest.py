import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from goodphotons_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "libftoracle.so")):
        build.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def L():
    from goodphotons_b200 import lib
    return lib.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle_bind import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle_bind import Reference
    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def gpu(L):
    if not L.available():
        pytest.skip("no CUDA device")
    return L
