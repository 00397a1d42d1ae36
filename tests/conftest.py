"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs the oracle against the reference's known answers and
the golden fixtures, the host-side packing logic, and the C-ABI export
check. `-m gpu` runs the CUDA library against the oracle and the fixtures.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import binding

    return binding.load()


@pytest.fixture(scope="session")
def cuda_lib():
    from stargaze_b200 import _lib

    return _lib.load()
