"""Shared fixtures. `gpu` marks tests that need a B200 (run with -m gpu)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    return np.load(GOLDEN / name)


def rel_l2(a, b):
    """||a - b||_2 / ||b||_2 over all components."""
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Orc
    return Orc()


@pytest.fixture(scope="session")
def ctx():
    from aster_b200.api import Context
    c = Context(0)
    yield c
    c.close()
