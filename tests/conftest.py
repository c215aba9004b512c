"""pytest configuration: the `gpu` marker and the checkers' build."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """The scalar oracle is test infrastructure; build it if this checkout
    has not (a few seconds with gcc)."""
    so = os.path.join(ROOT, "oracle", "liboracle_gasal.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       stdout=subprocess.DEVNULL)
    yield
