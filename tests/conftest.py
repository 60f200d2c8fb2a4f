"""Shared fixtures.  `gpu` marks tests that need a CUDA device (run with -m gpu)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def engine_lib():
    from fermiphasespace_b200 import build
    build.build_cuda()
    from fermiphasespace_b200 import engine
    return engine


@pytest.fixture()
def engine(engine_lib):
    eng = engine_lib.Engine(0)
    yield eng
    eng.close()
