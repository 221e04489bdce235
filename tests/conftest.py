import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def catch_approx(a, b, eps):
    """Catch v1.12 Approx (the reference's vendored catch.hpp:2841-2850):
    |a - b| < eps * (1 + max(|a|, |b|))."""
    return abs(a - b) < eps * (1.0 + max(abs(a), abs(b)))


@pytest.fixture(scope="session")
def kats():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")) as f:
        return json.load(f)
