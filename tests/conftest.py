"""Shared pytest set-up: repo root on sys.path, the `gpu` marker, library fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG = os.path.join(ROOT, "parode_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)  # the `ParODE` extension module lives here


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library on cuda:0)")


@pytest.fixture(scope="session")
def pb():
    """The CUDA library, initialised on every compute-capability-10 device."""
    import parode_b200 as pb

    pb.init()
    return pb
