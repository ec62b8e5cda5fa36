import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def ve():
    import helpers

    return helpers.package()


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import REF_LIB, Reference

    if not os.path.exists(REF_LIB):
        from oracle.oracle import build_ref

        build_ref()
    if not os.path.exists(REF_LIB):
        pytest.skip("reference octree library (oracle/_ref) not built: reference sources absent")
    return Reference()
