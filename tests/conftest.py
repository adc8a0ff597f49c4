"""Shared fixtures.

`-m "not gpu"` tests need only the host side: the tree/tape code, the C ABI
exports and the CPU oracle.  `-m gpu` tests call the CUDA path through the
C ABI and compare it with the oracle.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from libfive_b200 import build
    build.build(verbose=False)
    if subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")],
                      capture_output=True).returncode != 0:
        raise RuntimeError("oracle build failed")


_ensure_built()


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from libfive_b200 import ffi
    return ffi.load()


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.fail("gpu test run without a CUDA device")
    return True
