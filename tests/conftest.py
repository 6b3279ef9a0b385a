import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle, the CPU kernel-body harness and the solver library once."""
    for d in ("oracle", os.path.join("tests", "hostemu"), os.path.join("cism_b200", "csrc")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, d)], check=True)
    yield


@pytest.fixture(scope="session")
def ctx():
    from cism_b200 import solver

    c = solver.Context(0)
    yield c
    c.close()
