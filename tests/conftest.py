import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdynamap_b200.so")
    config.addinivalue_line(
        "markers", "first_b200_run: GPU tests of code that has not yet passed on a B200")


def pytest_collection_modifyitems(config, items):
    """Tests of code not yet run on a B200 go after all others, so that
    under -x a failure there cannot hide the results of the established
    tests; the allocation-free entry point's file (test_zz_*) stays last of
    all."""
    items.sort(key=lambda it: (os.path.basename(str(it.fspath)).startswith("test_zz"),
                               it.get_closest_marker("first_b200_run") is not None))


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.lib()
    pyoracle.set_threads(min(8, os.cpu_count() or 1))
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    from dynamap_b200 import abi
    lib = abi.load()  # raises if the CUDA library is missing: no fallback
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    return lib
