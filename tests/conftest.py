import os
import sys

import pytest

TESTS = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(TESTS)
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    import testlibs

    testlibs.build_all()


@pytest.fixture(scope="session")
def renderer():
    """One kt_context on cuda:0 for the GPU tests."""
    import kerrtracecpp2_b200 as kt

    r = kt.Renderer(0)
    yield r
    r.close()
