import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def triangulator():
    import gcdt_b200 as g
    t = g.Triangulator(max_points=1 << 21, max_segments=1 << 18)
    yield t
    t.close()
