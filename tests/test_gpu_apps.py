"""GPU tests of the command-line programs against the reference library:
nnp-predict (the reference tool's files and formats) and lammps-emulate
(n2p2b::InterfaceLammps driven like pair_style hdnnp: local atoms, ghost
images, a full neighbor list, getForces into local + ghost atoms, reverse
communication).  Energy 1e-10 relative, forces |dF| <= 1e-10 max(|F|,
rms F)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
POT = os.path.join(ROOT, "tests", "golden", "potentials", "h2o_52")
BIN = os.path.join(ROOT, "n2p2_b200", "bin")
SYM = {0: "H", 1: "O"}


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _write_input_data(path, box, pos, elem, energy=-1.0):
    with open(path, "w") as f:
        f.write("begin\ncomment synthetic water\n")
        for v in box:
            f.write("lattice %24.16E %24.16E %24.16E\n" % tuple(v))
        for r, e in zip(pos, elem):
            f.write("atom %24.16E %24.16E %24.16E %2s %24.16E %24.16E "
                    "%24.16E %24.16E %24.16E\n"
                    % (r[0], r[1], r[2], SYM[int(e)], 0.0, 0.0, 0.1, 0.2,
                       0.3))
        f.write("energy %24.16E\ncharge %24.16E\nend\n" % (energy, 0.0))


def _reference(box, pos, elem):
    from oracle.ref import RefModel
    ref = RefModel(POT)
    ref.set_structure(pos, elem, box)
    return ref.predict()


def _check(e, f, e0, f0):
    assert abs(e - e0) <= 1e-10 * abs(e0)
    tol = 1e-10 * np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    assert np.all(np.abs(f - f0) <= tol)


def test_nnp_predict_matches_reference(gpu, tmp_path):
    box, pos, elem = synth.water_box(64, 31)
    pos = pos + np.random.default_rng(4).normal(0, 0.1, pos.shape)
    for name in ("input.nn", "scaling.data", "weights.001.data",
                 "weights.008.data"):
        shutil.copy(os.path.join(POT, name), tmp_path / name)
    _write_input_data(tmp_path / "input.data", box, pos, elem, -123.0)
    r = subprocess.run([os.path.join(BIN, "nnp-predict"), "0"],
                       cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for name in ("energy.out", "nnatoms.out", "nnforces.out", "output.data",
                 "nnp-predict.log"):
        assert (tmp_path / name).exists()
    e0, f0 = _reference(box, pos, elem)
    rows = [ln.split() for ln in open(tmp_path / "energy.out")
            if not ln.startswith("#")]
    assert len(rows) == 1
    conf, natoms, eref, ennp = rows[0][:4]
    assert int(conf) == 1 and int(natoms) == len(elem)
    assert float(eref) == -123.0
    f = np.array([[float(x) for x in ln.split()[5:8]]
                  for ln in open(tmp_path / "nnforces.out")
                  if not ln.startswith("#")])
    fref = np.array([[float(x) for x in ln.split()[2:5]]
                     for ln in open(tmp_path / "nnforces.out")
                     if not ln.startswith("#")])
    assert np.allclose(fref, [0.1, 0.2, 0.3])
    _check(float(ennp), f, e0, f0)
    out = open(tmp_path / "output.data").read().split("\n")
    eline = [ln for ln in out if ln.startswith("energy")][0]
    assert abs(float(eline.split()[1]) - e0) <= 1e-10 * abs(e0)
    assert sum(ln.startswith("atom") for ln in out) == len(elem)


@pytest.mark.parametrize("cf", [(1.0, 1.0), (0.52917721, 27.211386)])
def test_interface_lammps_emulation(gpu, tmp_path, cf):
    """Local + ghost atoms through InterfaceLammps; the engine works in its
    own units (positions / cflength), the interface converts."""
    box, pos, elem = synth.water_box(32, 17)
    pos = pos + np.random.default_rng(5).normal(0, 0.1, pos.shape)
    L = box[0, 0]
    pos = np.mod(pos, L)
    cfl, cfe = cf
    _write_input_data(tmp_path / "input.data", box / cfl, pos / cfl, elem)
    r = subprocess.run([os.path.join(BIN, "lammps-emulate"), POT,
                        str(tmp_path / "input.data"), repr(cfl), repr(cfe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    e = float(lines[0].split()[1])
    f = np.array([[float(x) for x in ln.split()[2:5]] for ln in lines[1:]
                  if ln.startswith("force")])
    e0, f0 = _reference(box, pos, elem)
    # Engine units: E / cfenergy, F * cflength / cfenergy.
    _check(e * cfe, f * cfe / cfl, e0, f0)


_STEPS_CALLER = r'''
#include <cstdio>
#include "n2p2_b200.hpp"

static void dump(std::FILE* o, char const* tag, n2p2b::Structure const& s,
                 bool forces)
{
    std::fprintf(o, "%s %.17g\n", tag, s.energy);
    if (forces)
        for (double v : s.f) std::fprintf(o, "%.17g\n", v);
}

int main()
{
    n2p2b::Prediction p(0);
    p.initialize();
    p.setup();
    p.setupSymmetryFunctionGroups();
    p.readStructureFromFile("input.data");
    std::FILE* o = std::fopen("steps.out", "w");
    n2p2b::Structure s = p.structure;
    p.calculateSymmetryFunctionGroups(s, true);
    p.calculateAtomicNeuralNetworks(s, true);
    p.calculateEnergy(s);
    p.calculateForces(s);
    dump(o, "steps", s, true);
    n2p2b::Structure s2 = p.structure;
    p.evaluateNNP(s2);
    dump(o, "evaluateNNP", s2, true);
    n2p2b::Structure s3 = p.structure;
    p.evaluateNNP(s3, false, true);
    dump(o, "energy_dEdG", s3, false);
    n2p2b::Structure s4 = p.structure;
    p.evaluateNNP(s4, false, false);
    dump(o, "energy_only", s4, false);
    p.predict();
    dump(o, "predict", p.structure, true);
    std::fclose(o);
    return 0;
}
'''


def test_cpp_mode_steps_match_reference(gpu, tmp_path):
    """n2p2b::Prediction driven through the nnp::Mode evaluation steps
    (calculateSymmetryFunctionGroups -> calculateAtomicNeuralNetworks ->
    calculateEnergy -> calculateForces), evaluateNNP with and without forces
    and predict(): all equal to the reference library (energy 1e-10
    relative, forces 1e-10 of max(|F|, rms F)); the energy-only forms
    within 1e-12 of evaluateNNP's energy."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    lib = os.path.join(ROOT, "n2p2_b200")
    src = tmp_path / "steps.cpp"
    src.write_text(_STEPS_CALLER)
    exe = tmp_path / "steps"
    r = subprocess.run([gxx, "-std=c++17", "-O2",
                        "-I" + os.path.join(ROOT, "include"), str(src),
                        "-L" + lib, "-ln2p2b200", "-Wl,-rpath," + lib,
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    box, pos, elem = synth.water_box(64, 33)
    pos = pos + np.random.default_rng(6).normal(0, 0.1, pos.shape)
    for name in ("input.nn", "scaling.data", "weights.001.data",
                 "weights.008.data"):
        shutil.copy(os.path.join(POT, name), tmp_path / name)
    _write_input_data(tmp_path / "input.data", box, pos, elem)
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    blocks, cur = {}, None
    for ln in open(tmp_path / "steps.out"):
        t = ln.split()
        if len(t) == 2:
            cur = t[0]
            blocks[cur] = [float(t[1]), []]
        else:
            blocks[cur][1].append(float(t[0]))
    n = len(elem)
    e0, f0 = _reference(box, pos, elem)
    for tag in ("steps", "evaluateNNP", "predict"):
        e, f = blocks[tag][0], np.array(blocks[tag][1]).reshape(n, 3)
        _check(e, f, e0, f0)
    e1 = blocks["evaluateNNP"][0]
    for tag in ("energy_dEdG", "energy_only"):
        assert abs(blocks[tag][0] - e1) <= 1e-12 * abs(e1)
