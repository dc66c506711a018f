"""CPU checks of the C++ interface and the command-line programs: the
header compiles on its own, the programs are built and answer without a
GPU (usage text, clean error without a device)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "n2p2_b200", "bin")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_cpp_header_compiles(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "n2p2_b200.hpp"\n'
                   "int main() { n2p2b::Structure s; return (int)"
                   "s.numAtoms(); }\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only",
                        "-I" + os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_programs_built_and_print_usage():
    from n2p2_b200 import build
    build.build_apps()
    r = subprocess.run([os.path.join(BIN, "nnp-predict")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "USAGE" in r.stdout
    r = subprocess.run([os.path.join(BIN, "lammps-emulate")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "USAGE" in r.stderr


def test_input_data_round_trip(tmp_path):
    """Structure::readFromFile / writeToFile of the C++ interface."""
    (tmp_path / "in.data").write_text(
        "begin\ncomment two atoms\n"
        "lattice 10.0 0.0 0.0\nlattice 0.0 11.0 0.0\nlattice 0.0 0.0 12.0\n"
        "atom 1.0 2.0 3.0 H 0.5 0.0 0.1 0.2 0.3\n"
        "atom 4.0 5.0 6.0 O -0.5 0.0 0.4 0.5 0.6\n"
        "energy -7.25\ncharge 0.0\nend\n"
        "begin\ncomment second\natom 0 0 0 H 0 0 0 0 0\nenergy 1\n"
        "charge 0\nend\n")
    src = tmp_path / "rt.cpp"
    src.write_text(r'''
#include "n2p2_b200.hpp"
#include <cstdio>
int main(int, char** argv) {
    n2p2b::Structure s;
    if (!s.readFromFile(argv[1], 1)) return 3;
    if (s.numAtoms() != 1 || s.isPeriodic) return 4;
    if (!s.readFromFile(argv[1], 0)) return 5;
    s.energy = s.energyRef;
    std::FILE* f = std::fopen(argv[2], "w");
    s.writeToFile(f);
    std::fclose(f);
    return (s.numAtoms() == 2 && s.isPeriodic && s.box[1][1] == 11.0
            && s.chargeRef[1] == -0.5 && s.fRef[5] == 0.6
            && s.comment == "two atoms") ? 0 : 6;
}
''')
    exe = tmp_path / "rt"
    r = subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT,
                                                                "include"),
                        str(src), "-o", str(exe), "-L" + os.path.join(
                            ROOT, "n2p2_b200"), "-ln2p2b200",
                        "-Wl,-rpath," + os.path.join(ROOT, "n2p2_b200")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(tmp_path / "in.data"),
                        str(tmp_path / "out.data")], capture_output=True)
    assert r.returncode == 0
    out = (tmp_path / "out.data").read_text().split("\n")
    assert out[0] == "begin" and out[1] == "comment two atoms"
    assert out[2].split()[0] == "lattice"
    assert float([x for x in out if x.startswith("energy")][0].split()[1]) \
        == -7.25
