"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libaw_b200.so")


def _gpu_available() -> bool:
    try:
        from anchorwave_b200 import _lib
        return _lib.lib.aw_device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def restatement():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle
    try:
        return oracle.Reference()
    except FileNotFoundError as e:
        pytest.skip(str(e))


@pytest.fixture(scope="session")
def gpu():
    if not _gpu_available():
        pytest.fail("no CUDA device visible to libaw_b200.so (gpu tests must run on a GPU box)")
    from anchorwave_b200 import ksw2
    return ksw2
