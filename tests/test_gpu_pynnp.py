"""GPU tests of the pynnp-compatible classes: the reference's two pynnp
prediction examples (the Prediction shortcut, and the step-by-step Mode flow
with normalization and energy offsets) against the reference library.
Energy 1e-10 relative, forces |dF| <= 1e-10 max(|F|, rms F)."""
import os
import shutil

import numpy as np
import pytest

from n2p2_b200 import pynnp, synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials",
                   "h2o_52")
SYM = {0: "H", 1: "O"}


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _potential(d, normalized):
    for name in ("scaling.data", "weights.001.data", "weights.008.data"):
        shutil.copy(os.path.join(POT, name), d / name)
    text = open(os.path.join(POT, "input.nn")).read()
    if normalized:
        # Normalization (Mode::setupNormalization) and atomic energy offsets
        # (Mode::setupElements) on top of the same network.
        text += ("\nmean_energy -0.47\nconv_energy 2.5\nconv_length 1.3\n"
                 "atom_energy H -0.31\natom_energy O -1.7\n")
    (d / "input.nn").write_text(text)


def _structure(d, seed):
    box, pos, elem = synth.water_box(64, seed)
    pos = pos + np.random.default_rng(seed).normal(0, 0.1, pos.shape)
    with open(d / "input.data", "w") as fh:
        fh.write("begin\ncomment pynnp example\n")
        for v in box:
            fh.write("lattice %24.16E %24.16E %24.16E\n" % tuple(v))
        for r, e in zip(pos, elem):
            fh.write("atom %24.16E %24.16E %24.16E %2s %24.16E %24.16E "
                     "%24.16E %24.16E %24.16E\n"
                     % (r[0], r[1], r[2], SYM[int(e)], 0.0, 0.0, 0.0, 0.0,
                        0.0))
        fh.write("energy %24.16E\ncharge %24.16E\nend\n" % (-250.0, 0.0))
    return box, pos, elem


def _reference(d, box, pos, elem):
    from oracle.ref import RefModel
    ref = RefModel(str(d))
    ref.set_structure(pos, elem, box)
    return ref.predict()


def _check(e, f, e0, f0):
    assert abs(e - e0) <= 1e-10 * abs(e0)
    tol = 1e-10 * np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    assert np.all(np.abs(f - f0) <= tol)


def _forces(s):
    return np.array([a.f.r for a in s.atoms])


@pytest.mark.parametrize("normalized", [False, True])
def test_prediction_example(gpu, tmp_path, normalized):
    """Prediction(); setup(); readStructureFromFile(); predict()."""
    _potential(tmp_path, normalized)
    box, pos, elem = _structure(tmp_path, 41)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        p = pynnp.Prediction()
        p.setup()
        p.readStructureFromFile()
        p.predict()
        s = p.structure
        e0, f0 = _reference(tmp_path, box, pos, elem)
        _check(s.energy, _forces(s), e0, f0)
        assert s.energyRef == -250.0
        assert s.numAtomsPerElement == [128, 64]
        assert [p.elementMap[a.element] for a in s.atoms[:3]] == \
            [SYM[int(x)] for x in elem[:3]]
        if not normalized:
            esum = sum(a.energy for a in s.atoms)
            assert abs(esum - s.energy) <= 1e-10 * abs(s.energy)
        p.close()
    finally:
        os.chdir(cwd)


def test_mode_step_example_with_normalization(gpu, tmp_path):
    """The step-by-step Mode flow: setup steps, removeEnergyOffset,
    toNormalizedUnits, calculateNeighborList(getMaxCutoffRadius()),
    calculateSymmetryFunctionGroups, calculateAtomicNeuralNetworks,
    calculateEnergy, calculateForces, toPhysicalUnits, addEnergyOffset."""
    _potential(tmp_path, True)
    box, pos, elem = _structure(tmp_path, 43)
    d = str(tmp_path)
    m = pynnp.Mode()
    m.initialize()
    m.loadSettingsFile(os.path.join(d, "input.nn"))
    m.setupNormalization()
    assert m.useNormalization()
    mean, ce, cl = m.getMeanEnergy(), m.getConvEnergy(), m.getConvLength()
    assert (mean, ce, cl) == (-0.47, 2.5, 1.3)
    m.setupElementMap()
    m.setupElements()
    m.setupCutoff()
    m.setupSymmetryFunctions()
    m.setupSymmetryFunctionMemory()
    m.setupSymmetryFunctionCache()
    m.setupSymmetryFunctionGroups()
    m.setupNeuralNetwork()
    m.setupSymmetryFunctionScaling(os.path.join(d, "scaling.data"))
    m.setupNeuralNetworkWeights(os.path.join(d, "weights.%03zu.data"))
    m.setupSymmetryFunctionStatistics(True, True, True, False)
    s = pynnp.Structure()
    s.setElementMap(m.elementMap)
    s.readFromFile(os.path.join(d, "input.data"))
    m.removeEnergyOffset(s)
    s.toNormalizedUnits(mean, ce, cl)
    s.calculateNeighborList(m.getMaxCutoffRadius())
    m.calculateSymmetryFunctionGroups(s, True)
    assert s.atoms[0].numSymmetryFunctions == 52
    assert s.atoms[0].numNeighbors > 0
    m.calculateAtomicNeuralNetworks(s, True)
    m.calculateEnergy(s)
    m.calculateForces(s)
    s.toPhysicalUnits(mean, ce, cl)
    m.addEnergyOffset(s, False)
    m.addEnergyOffset(s, True)
    e0, f0 = _reference(tmp_path, box, pos, elem)
    _check(s.energy, _forces(s), e0, f0)
    assert abs(s.energyRef + 250.0) <= 1e-12 * 250.0
    m.close()
