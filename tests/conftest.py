"""Shared test setup.

Tests marked ``gpu`` need a CUDA device and call the product through the C ABI
(libwrk.so); everything else runs on the CPU: the oracle against the golden
fixtures and the reference's own code, host logic, and the C ABI's exports.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls libwrk.so through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    pyoracle.build()
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    import pyoracle

    if not os.path.exists(pyoracle.REF_LIB):
        pytest.skip("oracle/_ref/libref.so not built (needs the reference checkout)")
    return pyoracle.Reference()


@pytest.fixture(scope="session")
def wrk_lib():
    from offlinerenderer_b200 import build, wrk

    build.build()
    return wrk


@pytest.fixture(scope="session")
def gpu(wrk_lib):
    if wrk_lib.device_count() == 0:
        pytest.fail("gpu test selected but no CUDA device is visible")
    return wrk_lib


GOLDEN = os.path.join(ROOT, "tests", "golden")
