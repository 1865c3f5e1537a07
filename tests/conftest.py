import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    # one tuning table for the whole test session, subprocesses included:
    # measured by the first simulation created on the GPU, loaded by the rest
    if "NBODY_B200_TUNE_CACHE" not in os.environ:
        import tempfile
        os.environ["NBODY_B200_TUNE_CACHE"] = os.path.join(
            tempfile.gettempdir(), "nbody_b200_tests_%d_tune.bin" % os.getpid())
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
