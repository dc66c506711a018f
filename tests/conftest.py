import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

POT = os.path.join(ROOT, "tests", "golden", "potentials")
REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def pot_dir():
    return POT


def reference_tree_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "src", "libnnp"))
