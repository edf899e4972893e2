import os
import sys

import pytest

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for sub in ("sop-gpu_b200", "oracle", "tests"):
    p = os.path.join(REPO, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running check")


@pytest.fixture(scope="session")
def gpu_ctx():
    import sopb
    ctx = sopb.Context(0)
    yield ctx
    ctx.close()
