import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(autouse=True)
def _bounds_checked_build(request):
    """With TBMD_LIBRARY pointing at the bounds-checked build (libtbmd_checked.so), every GPU test
    ends with no kernel index recorded outside its array."""
    yield
    if request.node.get_closest_marker("gpu") is None or not os.environ.get("TBMD_LIBRARY"):
        return
    from threebodymdalgorithms_b200 import _lib
    checked, violations, site, index, size = _lib.bounds_report()
    if checked:
        assert violations == 0, f"{violations} index(es) outside their arrays; first: site {site}, {index} of {size}"
