"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and call the CUDA kernels through the
C ABI of libgdp.so; everything else runs on the CPU (oracle against the
reference and the golden vectors, host logic, library loading).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gmap-gsnap_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libgdp.so")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def gdplib():
    import gdp
    return gdp.load()


@pytest.fixture(scope="session")
def restatement():
    import oracle
    o = oracle.restatement()
    o.init(0)
    return o


@pytest.fixture(scope="session")
def reference():
    import oracle
    if not oracle.reference_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    o = oracle.reference()
    o.init(0)
    return o
