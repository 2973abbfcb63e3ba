"""Shared fixtures.  `gpu` marks tests that need a CUDA device and the
sm_100a library; everything else runs on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and delfem_b200/_lib/libdfm_b200.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def ctx():
    from delfem_b200 import lib
    c = lib.Context(0)
    yield c
    c.close()
