import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def fdtd():
    """The CUDA library; built in-tree if the .so is missing (nvcc is on the box)."""
    from fdtd_b200 import build_lib, grid
    if not os.path.exists(grid.LIB_PATH):
        build_lib.build()
    grid.load_library()
    return grid
