"""Shared fixtures.  `gpu` marks tests that need a CUDA device (run on the B200 box)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def restatement():
    from oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
