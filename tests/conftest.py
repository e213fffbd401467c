import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long GPU run (minutes of device time at most)")


def reference_available(nx, ny, nz):
    """The translated reference can be used if its sources are here or a
    prebuilt library for this grid travelled with the checkout."""
    from build_ref import REF_BLA, lib_path
    return os.path.isdir(REF_BLA) or os.path.exists(lib_path(nx, ny, nz))


@pytest.fixture
def need_ref():
    def _need(nx, ny, nz):
        if not reference_available(nx, ny, nz):
            pytest.skip("reference oracle neither buildable nor prebuilt for this grid")
    return _need
