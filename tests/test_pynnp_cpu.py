"""Host-side parts of the pynnp-compatible classes (no GPU): element map,
input.data reading and writing, energy offsets, unit conversions, Vec3D,
and the setup steps and queries of Mode / Prediction on a host-only
context."""
import os

import numpy as np
import pytest

from n2p2_b200 import pynnp, synth

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials",
                   "h2o_52")
SYM = {0: "H", 1: "O"}


def _write_input_data(path, box, pos, elem, energy=-7.5, comment="water"):
    rng = np.random.default_rng(1)
    f = rng.normal(size=pos.shape)
    with open(path, "w") as fh:
        fh.write(f"begin\ncomment {comment}\n")
        for v in box:
            fh.write("lattice %24.16E %24.16E %24.16E\n" % tuple(v))
        for r, e, fi in zip(pos, elem, f):
            fh.write("atom %24.16E %24.16E %24.16E %2s %24.16E %24.16E "
                     "%24.16E %24.16E %24.16E\n"
                     % (r[0], r[1], r[2], SYM[int(e)], 0.0, 0.0, *fi))
        fh.write("energy %24.16E\ncharge %24.16E\nend\n" % (energy, 0.0))
        fh.write("begin\ncomment second\nend\n")
    return f


def _host_mode():
    m = pynnp.Mode(device=-1)
    m.initialize()
    m.loadSettingsFile(os.path.join(POT, "input.nn"))
    m.setupNormalization()
    m.setupElementMap()
    m.setupElements()
    m.setupCutoff()
    m.setupSymmetryFunctions()
    m.setupSymmetryFunctionMemory()
    m.setupSymmetryFunctionCache()
    m.setupSymmetryFunctionGroups()
    m.setupNeuralNetwork()
    m.setupSymmetryFunctionScaling(os.path.join(POT, "scaling.data"))
    m.setupNeuralNetworkWeights(os.path.join(POT, "weights.%03zu.data"))
    m.setupSymmetryFunctionStatistics(True, True, True, False)
    return m


def test_mode_setup_steps_and_queries():
    m = _host_mode()
    em = m.elementMap
    assert em.size() == 2 and em[0] == "H" and em["O"] == 1
    assert list(em) == ["H", "O"]
    with pytest.raises(KeyError):
        em["C"]
    assert m.getMaxCutoffRadius() == 12.0
    assert not m.useNormalization()
    assert (m.getMeanEnergy(), m.getConvEnergy(), m.getConvLength()) == \
        (0.0, 1.0, 1.0)
    assert m.settingsKeywordExists("cutoff_type")
    assert not m.settingsKeywordExists("mean_energy")
    assert m.settingsGetValue("elements") == "H O"
    m.close()


def test_structure_read_write_round_trip(tmp_path):
    box, pos, elem = synth.water_box(16, 3)
    f = _write_input_data(tmp_path / "input.data", box, pos, elem)
    s = pynnp.Structure()
    s.setElementMap(pynnp.ElementMap(["H", "O"]))
    s.readFromFile(str(tmp_path / "input.data"))
    assert s.numAtoms == 48 and s.numAtomsPerElement == [32, 16]
    assert s.numElementsPresent == 2
    assert s.isPeriodic and not s.isTriclinic
    assert s.comment == "water"
    assert s.energyRef == -7.5
    assert np.isclose(s.volume, abs(np.linalg.det(box)))
    a = s.atoms[5]
    assert a.index == 5 and a.element == int(elem[5])
    assert a.r.r == list(pos[5]) and a.fRef.r == list(f[5])
    assert [v.r for v in s.box] == [list(v) for v in box]
    s.writeToFile(str(tmp_path / "out.data"))
    t = pynnp.Structure()
    t.setElementMap(pynnp.ElementMap(["H", "O"]))
    t.readFromFile(str(tmp_path / "out.data"))
    assert np.array_equal(t._r, s._r) and np.array_equal(t._fRef, s._fRef)
    assert t.energyRef == s.energyRef and np.array_equal(t._box, s._box)
    with pytest.raises(KeyError):
        u = pynnp.Structure()
        u.setElementMap(pynnp.ElementMap(["H"]))
        u.readFromFile(str(tmp_path / "input.data"))


def test_units_and_offsets(tmp_path):
    box, pos, elem = synth.water_box(8, 4)
    _write_input_data(tmp_path / "input.data", box, pos, elem, energy=3.0)
    s = pynnp.Structure()
    s.setElementMap(pynnp.ElementMap(["H", "O"]))
    s.readFromFile(str(tmp_path / "input.data"))
    r0, f0, e0, v0 = s._r.copy(), s._fRef.copy(), s.energyRef, s.volume
    mean, ce, cl = -0.25, 3.0, 2.0
    s.toNormalizedUnits(mean, ce, cl)
    assert np.array_equal(s._r, r0 * cl)
    assert np.allclose(s._fRef, f0 * ce / cl)
    assert np.isclose(s.energyRef, (e0 - 24 * mean) * ce)
    assert np.isclose(s.volume, v0 * cl ** 3)
    s.toPhysicalUnits(mean, ce, cl)
    assert np.array_equal(s._r, r0)
    assert np.allclose(s._fRef, f0) and np.isclose(s.energyRef, e0)
    m = _host_mode()
    m.removeEnergyOffset(s)
    m.addEnergyOffset(s)
    assert s.energyRef == e0                # h2o_52 has no atom_energy
    m.close()


def test_vec3d():
    a, b = pynnp.Vec3D(1.0, 2.0, 2.0), pynnp.Vec3D(0.0, 1.0, 0.0)
    assert a.norm() == 3.0 and a.norm2() == 9.0 and a * b == 2.0
    assert (a + b).r == [1.0, 3.0, 2.0] and (2.0 * b).r == [0.0, 2.0, 0.0]
    assert a.cross(b).r == [-2.0, 0.0, 1.0]
    a -= b
    assert a.r == [1.0, 1.0, 2.0]
    a[2] = 5.0
    assert a[2] == 5.0


def test_prediction_host_setup_and_read(tmp_path):
    for name in ("input.nn", "scaling.data", "weights.001.data",
                 "weights.008.data"):
        (tmp_path / name).write_bytes(open(os.path.join(POT, name),
                                           "rb").read())
    box, pos, elem = synth.water_box(8, 5)
    _write_input_data(tmp_path / "input.data", box, pos, elem)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        p = pynnp.Prediction(device=-1)
        p.setup()
        p.readStructureFromFile()
        s = p.structure
        assert s.numAtoms == 24 and s.energyRef == -7.5
        with pytest.raises(Exception):
            p.predict()                      # no GPU in a host context
        p.close()
    finally:
        os.chdir(cwd)


def test_structure_parser_edge_cases():
    """begin arguments, comment text, open (non-periodic) structures, a
    triclinic cell and the reference's errors for malformed input."""
    em = pynnp.ElementMap(["H", "O"])
    s = pynnp.Structure()
    s.setElementMap(em)
    s.readFromLines(["begin set=train", "comment  two  words ",
                     "atom 0 0 0 O 0.5 0 1 2 3",
                     "atom 1 0 0 H -0.25 0 0 0 0",
                     "energy -1.5", "charge 0.25", "end"])
    assert s.sampleType == 1 and not s.isPeriodic
    assert s.comment == " two  words "
    assert s.numAtomsPerElement == [1, 1] and s.chargeRef == 0.25
    assert [a.chargeRef for a in s.atoms] == [0.5, -0.25]
    assert s.atoms[0].fRef.r == [1.0, 2.0, 3.0]
    t = pynnp.Structure()
    t.setElementMap(em)
    t.readFromLines(["begin", "lattice 10 0 0", "lattice 1 10 0",
                     "lattice 0 0 10", "atom 0 0 0 H 0 0 0 0 0", "end"])
    assert t.isPeriodic and t.isTriclinic and np.isclose(t.volume, 1000.0)
    for bad in (["atom 0 0 0 H 0 0 0 0 0", "end"],
                ["begin set=other", "end"],
                ["begin", "lattice 1 0 0", "end"],
                ["begin", "velocity 0 0 0", "end"]):
        u = pynnp.Structure()
        u.setElementMap(em)
        with pytest.raises(RuntimeError):
            u.readFromLines(bad)


def test_mode_steps_need_symmetry_functions_first():
    m = _host_mode()
    s = pynnp.Structure()
    s.setElementMap(m.elementMap)
    s.readFromLines(["begin", "atom 0 0 0 H 0 0 0 0 0", "end"])
    with pytest.raises(RuntimeError):
        m.calculateAtomicNeuralNetworks(s, True)
    with pytest.raises(RuntimeError):
        m.calculateSymmetryFunctionGroups(s, True)   # no neighbor list yet
    s.calculateNeighborList(1.0)
    with pytest.raises(ValueError):
        m.calculateSymmetryFunctionGroups(s, True)   # cutoff below 12
    m.close()
