import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: longer CPU case")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.load()
    return pyoracle


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_expectations.json")) as fh:
        return json.load(fh)
