import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


import json

import pytest


@pytest.fixture
def record(request):
    """Measured errors of a test, appended as one JSON line to the file named
    by the PARITY_LOG environment variable (nothing is written without it)."""
    out = {}
    yield out
    path = os.environ.get("PARITY_LOG")
    if path and out:
        with open(path, "a") as f:
            f.write(json.dumps({"test": request.node.nodeid, **out}) + "\n")
