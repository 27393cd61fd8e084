"""Test configuration: the `gpu` marker and shared fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "rust-pricing-library_b200")):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")


@pytest.fixture(scope="session")
def oracle():
    import helpers
    return helpers.oracle()


@pytest.fixture(scope="session")
def engine():
    """The engine library; on a GPU machine it must load (no fallback)."""
    from rust_pricing_b200 import _native
    return _native.library()
