import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the device path")
    # the in-tree library must exist and be built from the sources beside it;
    # (re)build it once if it is missing or stale, then prove it
    from hmat_lib_b200 import abi, build
    stale = not os.path.exists(abi.lib_path())
    if not stale:
        # probed in a child process: a library loaded here could not be
        # replaced by a rebuild within this process
        import subprocess
        probe = subprocess.run(
            [sys.executable, "-c",
             "import ctypes as C, sys; l = C.CDLL(sys.argv[1]); "
             "l.hodlr_b200_version.restype = C.c_char_p; print(l.hodlr_b200_version().decode())",
             abi.lib_path()], capture_output=True, text=True)
        stale = probe.returncode != 0 or \
            probe.stdout.strip().rsplit(" ", 1)[-1] != build.source_hash()
    if stale:
        build.build()
    abi.check_source_hash(abi.load())


@pytest.fixture(scope="session")
def lib():
    from hmat_lib_b200 import abi
    return abi.load()


@pytest.fixture(scope="session")
def ref_available():
    from oracle import ref_lib
    return ref_lib.available()
