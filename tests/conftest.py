import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_v10.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle module, with the library's canonical reduction layout."""
    from oracle import oracle as om
    from mnhack8_b200 import _lib

    lay = _lib.layout(128)
    om.set_layout(0, 0, 0, lay["kf"])   # 0: the per-N tile shape, as the library
    return om
