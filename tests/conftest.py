import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "cpu-renderer_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def crgpu():
    import crgpu as m
    return m


@pytest.fixture(scope="session")
def gpu(crgpu):
    """The GPU tests never skip: on a box without a device they fail loudly."""
    n = crgpu.device_count()
    assert n >= 1, "no CUDA device visible"
    return 0


@pytest.fixture(scope="session")
def ref():
    import refimpl
    if not refimpl.available():
        pytest.skip("reference library oracle/_ref/libcr_ref.so not built here")
    return refimpl


GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    path = os.path.join(GOLDEN, name)
    return np.load(path) if os.path.exists(path) else None
