"""Shared pytest configuration.

Marker ``gpu``: needs a CUDA device (run with ``-m gpu`` on a B200 box); every
other test runs on a CPU-only machine.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def cblib():
    """The product's native library, built in-tree if needed."""
    from cast_simulator_b200 import build as B

    B.build()
    from cast_simulator_b200 import _lib

    return _lib.lib()
