import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Build the oracle (checker) and the engine library once per session."""
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)
    subprocess.run(["make", "-C", os.path.join(ROOT, "specrel_b200"), "-s", "-j8"], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return True


@pytest.fixture(scope="session")
def engine():
    import specrel_b200 as sr
    e = sr.Engine(0)
    yield e
    e.close()
