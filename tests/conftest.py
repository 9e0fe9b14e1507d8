import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the device path")
    # the in-tree library must exist; build it once if it is missing
    from hmat_lib_b200 import abi
    if not os.path.exists(abi.lib_path()):
        from hmat_lib_b200 import build
        build.build()


@pytest.fixture(scope="session")
def lib():
    from hmat_lib_b200 import abi
    return abi.load()


@pytest.fixture(scope="session")
def ref_available():
    from oracle import ref_lib
    return ref_lib.available()
