import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: several seconds of CPU work in the oracle")


@pytest.fixture(scope="session")
def ctx():
    import mobileraytracer_b200 as m
    c = m.Context(0)
    yield c
    c.close()
