"""Shared test setup: import paths, the `gpu` marker, device helpers."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "aocl-fftz_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")


@pytest.fixture(scope="session")
def gpulib():
    import aoclfftz_b200
    return aoclfftz_b200.load()
