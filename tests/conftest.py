"""Shared pytest configuration: the `gpu` marker and repo-root imports."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_sessionstart(session):
    # the library under test is the one built from this tree: rebuild it when
    # its embedded source hash differs (a no-op when it is up to date)
    from pedalsky_b200 import build
    build.build()


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def oracle_noise(oracle):
    return oracle.bake_noise()
