"""The LAMMPS pair style compiles unchanged against this library (CPU).

LAMMPS's pair_style hdnnp -- the reference's own
src/interface/LAMMPS/src/ML-HDNNP/pair_hdnnp.{h,cpp}, compiled where it lies,
not copied -- is built against include/InterfaceLammps.h (the drop-in
nnp::InterfaceLammps with its `log` member) and a single-rank stand-in for
the LAMMPS headers it includes (tests/lammps_stub/include), and linked with
n2p2_b200/libn2p2b200.so into tests/lammps_stub/_build/lammps_pair_hdnnp.
The GPU test tests/test_gpu_lammps_dropin.py runs that program.
"""
import os
import subprocess

import pytest

from conftest import REFERENCE, ROOT, reference_tree_available

STUB = os.path.join(ROOT, "tests", "lammps_stub")


@pytest.mark.skipif(not reference_tree_available(),
                    reason="reference tree (pair_hdnnp.cpp) not present")
def test_pair_hdnnp_compiles_and_links_unchanged():
    r = subprocess.run(["make", "-C", STUB, f"N2P2_REFERENCE={REFERENCE}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "warning" not in r.stderr.lower(), r.stderr
    assert os.access(os.path.join(STUB, "_build", "lammps_pair_hdnnp"),
                     os.X_OK)
