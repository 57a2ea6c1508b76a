"""Shared test configuration.

Markers: tests that need a CUDA device are marked `gpu`; everything else runs on CPU.
The repository root is put on sys.path so tests can import orkan_b200 (the product
binding), oracle (the CPU checker) and the test helpers.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref5():
    from oracle import ref
    if not ref.available(5):
        pytest.skip("oracle/_ref/liborkan_ref_t5.so not built (needs the reference sources)")
    return ref.RefLib(5)


@pytest.fixture(scope="session")
def ref3():
    from oracle import ref
    if not ref.available(3):
        pytest.skip("oracle/_ref/liborkan_ref_t3.so not built (needs the reference sources)")
    return ref.RefLib(3)


@pytest.fixture(scope="session")
def ork5():
    import orkan_b200
    return orkan_b200.load(5)


@pytest.fixture(scope="session")
def ork3():
    import orkan_b200
    return orkan_b200.load(3)
