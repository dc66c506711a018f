import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

POT = os.path.join(ROOT, "tests", "golden", "potentials")
REF_EXAMPLES = os.path.join(ROOT, "tests", "golden", "ref_examples")
# The reference source tree (only needed to regenerate fixtures and for the
# host-setup comparisons that read the reference's own example directories).
REFERENCE = os.environ.get("N2P2_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def pot_dir():
    return POT


def reference_tree_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "src", "libnnp"))


def ref_example(name):
    """One of the reference's nnp-predict examples as committed under
    tests/golden/ref_examples: (directory, box or None, positions, element
    symbols, golden energy, golden forces[N, 3])."""
    import numpy as np
    from oracle.ref import read_input_data
    d = os.path.join(REF_EXAMPLES, name)
    fr = read_input_data(os.path.join(d, "input.data"))[0]
    with open(os.path.join(d, "golden.txt")) as fh:
        energy = float(fh.readline().split()[1])
        forces = np.array([[float(x) for x in ln.split()] for ln in fh
                           if ln.strip()])
    return d, fr["box"], fr["pos"], fr["sym"], energy, forces
