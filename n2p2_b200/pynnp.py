"""pynnp-compatible classes for prediction scripts (src/pynnp/*.pyx).

Scripts written against the reference's Cython module switch by replacing
``import pynnp`` with ``from n2p2_b200 import pynnp``: ``Mode`` (setup steps,
the evaluation steps on a ``Structure``, energy offsets, normalization
queries, ``elementMap``), ``Prediction`` (``setup``,
``readStructureFromFile``, ``predict``, ``structure``), ``Structure``,
``Atom``, ``Vec3D`` and ``ElementMap`` keep pynnp's names and meanings
(src/pynnp/Mode.pyx:17-110, Prediction.pyx, Structure.pyx, Atom.pyx,
Vec3D.pyx, ElementMap.pyx).  The work runs in the library on the GPU through
``n2p2_b200.mode``; this module only keeps the host-side structure and its
units.

Units follow the reference: a structure is in physical units until
``toNormalizedUnits`` and back after ``toPhysicalUnits``; each evaluation
step leaves its results in the structure's current units (energies without
offsets, as ``Mode::calculateEnergy`` leaves them; ``addEnergyOffset`` adds
them).  Differences: ``calculateNeighborList`` only records the cutoff (the
list is built on the device by ``calculateSymmetryFunctionGroups``, which
needs a cutoff of at least ``getMaxCutoffRadius()``); periodic positions are
wrapped into the cell on the device as ``Structure::remap`` does, while
``atom.r`` keeps the values as read; neighbor objects, the log and 4G
(charge) networks are not provided.
"""
from __future__ import annotations

import numpy as np

from . import mode as _mode


class ElementMap:
    """nnp::ElementMap: index <-> symbol in the potential's element order."""

    def __init__(self, symbols=()):
        self._symbols = list(symbols)

    def __getitem__(self, item):
        if isinstance(item, (int, np.integer)):
            if item < 0 or item >= len(self._symbols):
                raise IndexError(item)
            return self._symbols[int(item)]
        if isinstance(item, str):
            return self.index(item)
        raise NotImplementedError

    def __len__(self):
        return len(self._symbols)

    def size(self):
        return len(self._symbols)

    def index(self, symbol):
        try:
            return self._symbols.index(symbol)
        except ValueError:
            raise KeyError(f"element {symbol!r} not in the element map")

    def symbol(self, index):
        return self[index]


class Vec3D:
    """nnp::Vec3D over three doubles (a view into its structure's arrays
    when it belongs to an atom or a box)."""

    def __init__(self, x=None, y=None, z=None, _view=None):
        if _view is not None:
            self._v = _view
        elif isinstance(x, Vec3D):
            self._v = x._v.copy()
        else:
            self._v = np.array([x or 0.0, y or 0.0, z or 0.0], dtype=float)

    @property
    def r(self):
        return [float(c) for c in self._v]

    @r.setter
    def r(self, value):
        self._v[:] = value

    def __getitem__(self, i):
        return float(self._v[i])

    def __setitem__(self, i, value):
        self._v[i] = value

    def __str__(self):
        return "{:24.16E} {:24.16E} {:24.16E}".format(*self._v)

    def __iadd__(self, v):
        self._v += v._v
        return self

    def __isub__(self, v):
        self._v -= v._v
        return self

    def __imul__(self, a):
        self._v *= a
        return self

    def __itruediv__(self, a):
        self._v /= a
        return self

    def __add__(self, v):
        return Vec3D(*(self._v + v._v))

    def __sub__(self, v):
        return Vec3D(*(self._v - v._v))

    def __neg__(self):
        return Vec3D(*(-self._v))

    def __mul__(self, other):
        if isinstance(other, Vec3D):
            return float(self._v @ other._v)
        return Vec3D(*(self._v * other))

    __rmul__ = __mul__

    def __truediv__(self, a):
        return Vec3D(*(self._v / a))

    def norm(self):
        return float(np.sqrt(self._v @ self._v))

    def norm2(self):
        return float(self._v @ self._v)

    def normalize(self):
        self._v /= self.norm()
        return self

    def cross(self, v):
        return Vec3D(*np.cross(self._v, v._v))


class Atom:
    """nnp::Atom of a Structure (a view: changes write through)."""

    def __init__(self, structure, i):
        self._s = structure
        self._i = i

    index = property(lambda a: a._i)
    indexStructure = property(lambda a: a._s.index)
    tag = property(lambda a: a._i)
    element = property(lambda a: int(a._s._elem[a._i]))
    r = property(lambda a: Vec3D(_view=a._s._r[a._i]))
    f = property(lambda a: Vec3D(_view=a._s._f[a._i]))
    fRef = property(lambda a: Vec3D(_view=a._s._fRef[a._i]))
    hasNeighborList = property(lambda a: a._s.hasNeighborList)
    hasSymmetryFunctions = property(lambda a: a._s.hasSymmetryFunctions)
    hasSymmetryFunctionDerivatives = property(
        lambda a: a._s.hasSymmetryFunctionDerivatives)

    @property
    def energy(self):
        return float(self._s._energyAtom[self._i])

    @energy.setter
    def energy(self, value):
        self._s._energyAtom[self._i] = value

    @property
    def charge(self):
        return float(self._s._charge[self._i])

    @property
    def chargeRef(self):
        return float(self._s._chargeRef[self._i])

    @property
    def numNeighbors(self):
        c = self._s._numNeighbors
        return 0 if c is None else int(c[self._i])

    @property
    def numSymmetryFunctions(self):
        g = self._s._G
        return 0 if g is None else int(self._s._numSF[self.element])

    @property
    def G(self):
        if self._s._G is None:
            return []
        return [float(x) for x in
                self._s._G[self._i, :self._s._numSF[self.element]]]

    @property
    def dEdG(self):
        if self._s._dEdG is None:
            return []
        return [float(x) for x in
                self._s._dEdG[self._i, :self._s._numSF[self.element]]]


class Structure:
    """nnp::Structure (input.data format, Structure.cpp:142-271)."""

    def __init__(self, empty=False):
        self.elementMap = ElementMap()
        self.reset()

    def reset(self):
        self._token = object()          # identifies this content to Mode
        self.index = 0
        self.comment = ""
        self.isPeriodic = False
        self.isTriclinic = False
        self.hasNeighborList = False
        self.hasSymmetryFunctions = False
        self.hasSymmetryFunctionDerivatives = False
        self.energy = 0.0
        self.energyRef = 0.0
        self.charge = 0.0
        self.chargeRef = 0.0
        self.volume = 0.0
        self.sampleType = 0
        self._box = np.zeros((3, 3))
        self._symbols = []
        self._elem = np.zeros(0, dtype=np.int32)
        self._r = np.zeros((0, 3))
        self._f = np.zeros((0, 3))
        self._fRef = np.zeros((0, 3))
        self._energyAtom = np.zeros(0)
        self._charge = np.zeros(0)
        self._chargeRef = np.zeros(0)
        self._numNeighbors = None
        self._G = self._dEdG = None
        self._numSF = None
        self._cutoff = None
        # Normalization applied by toNormalizedUnits (None: physical units)
        # and the physical positions and box it started from.
        self._norm = None
        self._phys = None

    def setElementMap(self, elementMap):
        self.elementMap = elementMap

    # ---- input.data --------------------------------------------------------
    def readFromFile(self, fileName="input.data"):
        """First configuration of the file."""
        lines = []
        with open(fileName) as fh:
            for line in fh:
                w = line.split()
                if not lines and (not w or w[0] != "begin"):
                    raise RuntimeError('ERROR: Unexpected file content, '
                                       'expected "begin" keyword.\n')
                lines.append(line.rstrip("\n"))
                if w and w[0] == "end":
                    break
        if not lines:
            raise RuntimeError(f'ERROR: No configuration in "{fileName}".\n')
        self.readFromLines(lines)

    def readFromLines(self, lines):
        if not lines or not lines[0].split() or lines[0].split()[0] != "begin":
            raise RuntimeError('ERROR: Unexpected line content, expected '
                               '"begin" keyword.\n')
        box, r, sym, qref, fref = [], [], [], [], []
        for line in lines:
            w = line.split()
            if not w:
                continue
            k = w[0]
            if k == "begin":
                for word in w[1:]:
                    if word == "set=train":
                        self.sampleType = 1
                    elif word == "set=test":
                        self.sampleType = 2
                    else:
                        raise RuntimeError("ERROR: Unknown keyword in "
                                           "structure specification, check "
                                           '"begin" arguments.\n')
            elif k == "comment":
                p = line.find("comment")
                self.comment = line[:p] + line[p + len("comment") + 1:]
            elif k == "lattice":
                if len(box) > 2:
                    raise RuntimeError("ERROR: Too many box vectors.\n")
                box.append([float(x) for x in w[1:4]])
            elif k == "atom":
                r.append([float(x) for x in w[1:4]])
                sym.append(w[4])
                qref.append(float(w[5]))
                fref.append([float(x) for x in w[7:10]])
            elif k == "energy":
                self.energyRef = float(w[1])
            elif k == "charge":
                self.chargeRef = float(w[1])
            elif k == "end":
                break
            else:
                raise RuntimeError("ERROR: Unexpected file content, unknown "
                                   f'keyword "{k}".\n')
        if len(box) not in (0, 3):
            raise RuntimeError("ERROR: Strange number of box vectors.\n")
        n = len(r)
        self._token = object()
        self._symbols = sym
        self._elem = np.array([self.elementMap[s] for s in sym],
                              dtype=np.int32)
        self._r = np.array(r, dtype=float).reshape(n, 3)
        self._fRef = np.array(fref, dtype=float).reshape(n, 3)
        self._f = np.zeros((n, 3))
        self._energyAtom = np.zeros(n)
        self._charge = np.zeros(n)
        self._chargeRef = np.array(qref, dtype=float)
        if box:
            self._box = np.array(box, dtype=float)
            self.isPeriodic = True
            off = self._box[~np.eye(3, dtype=bool)]
            self.isTriclinic = bool(np.any(off > np.finfo(float).tiny))
            self.volume = float(abs(np.linalg.det(self._box)))

    def writeToFile(self, fileName="output.data", ref=True, append=False):
        """Structure::writeToFile (Structure.cpp:1449-1531): reference or
        predicted energy and forces."""
        e = self.energyRef if ref else self.energy
        f = self._fRef if ref else self._f
        q = self._chargeRef if ref else self._charge
        with open(fileName, "a" if append else "w") as fh:
            fh.write("begin\n")
            fh.write(f"comment {self.comment}\n")
            if self.isPeriodic:
                for v in self._box:
                    fh.write("lattice {:24.16E} {:24.16E} {:24.16E}\n"
                             .format(*v))
            for i in range(self.numAtoms):
                fh.write("atom {:24.16E} {:24.16E} {:24.16E} {:>2s} {:24.16E} "
                         "{:24.16E} {:24.16E} {:24.16E} {:24.16E}\n".format(
                             *self._r[i], self._symbols[i], q[i], 0.0,
                             *f[i]))
            fh.write("energy {:24.16E}\n".format(e))
            fh.write("charge {:24.16E}\n".format(
                self.chargeRef if ref else self.charge))
            fh.write("end\n")

    # ---- neighbor list and units ------------------------------------------
    def calculateNeighborList(self, cutoffRadius):
        self._cutoff = float(cutoffRadius)
        self.hasNeighborList = True

    def clearNeighborList(self):
        self._cutoff = None
        self._numNeighbors = None
        self.hasNeighborList = False

    def remap(self):
        """Periodic positions are wrapped into the cell on the device at the
        next evaluation (Structure::remap's arithmetic); nothing to do on
        the host."""

    def toNormalizedUnits(self, meanEnergy, convEnergy, convLength,
                          convCharge=1.0):
        """Structure::toNormalizedUnits + Atom::toNormalizedUnits
        (Structure.cpp:1249-1276, Atom.cpp:78-120)."""
        self._phys = (self._r.copy(), self._box.copy())
        self._norm = (meanEnergy, convEnergy, convLength, convCharge)
        n = self.numAtoms
        self._box *= convLength
        self.energyRef = (self.energyRef - n * meanEnergy) * convEnergy
        self.energy = (self.energy - n * meanEnergy) * convEnergy
        self.chargeRef *= convCharge
        self.charge *= convCharge
        self.volume *= convLength ** 3
        self._r *= convLength
        self._f *= convEnergy / convLength
        self._fRef *= convEnergy / convLength
        self._energyAtom *= convEnergy
        self._charge *= convCharge
        self._chargeRef *= convCharge
        if self._dEdG is not None:
            self._dEdG *= convEnergy

    def toPhysicalUnits(self, meanEnergy, convEnergy, convLength,
                        convCharge=1.0):
        """Structure::toPhysicalUnits + Atom::toPhysicalUnits
        (Structure.cpp:1278-1305)."""
        n = self.numAtoms
        self._box /= convLength
        self.energyRef = self.energyRef / convEnergy + n * meanEnergy
        self.energy = self.energy / convEnergy + n * meanEnergy
        self.chargeRef /= convCharge
        self.charge /= convCharge
        self.volume /= convLength ** 3
        self._r /= convLength
        self._f /= convEnergy / convLength
        self._fRef /= convEnergy / convLength
        self._energyAtom /= convEnergy
        self._charge /= convCharge
        self._chargeRef /= convCharge
        if self._dEdG is not None:
            self._dEdG /= convEnergy
        if self._phys is not None and self._norm == (
                meanEnergy, convEnergy, convLength, convCharge):
            # Back to the exact positions and box that were normalized.
            r0, b0 = self._phys
            if np.allclose(r0, self._r, rtol=1e-14, atol=0.0):
                self._r[:] = r0
            if np.allclose(b0, self._box, rtol=1e-14, atol=0.0):
                self._box[:] = b0
        self._phys = None
        self._norm = None

    # ---- properties --------------------------------------------------------
    @property
    def numAtoms(self):
        return len(self._symbols)

    @property
    def numElements(self):
        return self.elementMap.size()

    @property
    def numAtomsPerElement(self):
        return [int(np.count_nonzero(self._elem == e))
                for e in range(self.numElements)]

    @property
    def numElementsPresent(self):
        return sum(1 for c in self.numAtomsPerElement if c > 0)

    @property
    def box(self):
        return [Vec3D(_view=self._box[i]) for i in range(3)]

    @property
    def atoms(self):
        return [Atom(self, i) for i in range(self.numAtoms)]

    # ---- device exchange (used by Mode) ------------------------------------
    def _physical_positions(self):
        """Positions and box in physical units for the library."""
        if self._norm is None:
            return self._r, (self._box if self.isPeriodic else None)
        c = self._norm[2]
        r0, b0 = self._phys
        r = r0 if np.array_equal(r0 * c, self._r) else self._r / c
        b = b0 if np.array_equal(b0 * c, self._box) else self._box / c
        return r, (b if self.isPeriodic else None)

    def _energy_scale(self):
        """(mean energy, energy factor) from physical to current units."""
        if self._norm is None:
            return 0.0, 1.0
        return self._norm[0], self._norm[1]


class Mode:
    """nnp::Mode (src/pynnp/Mode.pyx:17-110) over the library."""

    def __init__(self, device: int = 0):
        self._m = _mode.Mode(device)
        self._generic = False
        self._settings_file = None
        self._uploaded = None

    # ---- setup -------------------------------------------------------------
    def initialize(self):
        """Mode::initialize writes the reference's banner only."""

    def loadSettingsFile(self, fileName="input.nn"):
        self._m.load_settings_file(fileName)
        self._settings_file = fileName

    def setupGeneric(self):
        if not self._generic:
            self._m.setup_generic()
            self._generic = True

    # The reference's setupGeneric runs these steps in this order
    # (Mode.cpp:212-236); the library runs them together.
    setupNormalization = setupGeneric
    setupElementMap = setupGeneric
    setupElements = setupGeneric
    setupCutoff = setupGeneric
    setupSymmetryFunctions = setupGeneric
    setupSymmetryFunctionGroups = setupGeneric
    setupNeuralNetwork = setupGeneric

    def setupSymmetryFunctionMemory(self, verbose=False):
        self.setupGeneric()

    def setupSymmetryFunctionCache(self, verbose=False):
        self.setupGeneric()

    def setupSymmetryFunctionScalingNone(self):
        self.setupGeneric()
        self._m.setup_symmetry_function_scaling_none()

    def setupSymmetryFunctionScaling(self, fileName="scaling.data"):
        self.setupGeneric()
        self._m.setup_symmetry_function_scaling(fileName)

    def setupNeuralNetworkWeights(self, fileNameFormat="weights.%03zu.data"):
        self._m.setup_neural_network_weights(fileNameFormat)

    def setupSymmetryFunctionStatistics(self, collectStatistics,
                                        collectExtrapolationWarnings,
                                        writeExtrapolationWarnings,
                                        stopOnExtrapolationWarnings):
        """Extrapolation warnings as the reference counts, writes and stops
        on them.  collectStatistics (per-SF statistics for the training
        tools, which pynnp offers no way to read) is accepted and not
        collected."""
        self._m.setup_symmetry_function_statistics(
            False, collectExtrapolationWarnings,
            writeExtrapolationWarnings, stopOnExtrapolationWarnings)

    # ---- queries -----------------------------------------------------------
    @property
    def elementMap(self):
        return ElementMap(self._m.elements)

    def getMaxCutoffRadius(self):
        return self._m.get_max_cutoff_radius()

    def _units(self):
        return self._m.unit_conversion()

    def useNormalization(self):
        return self._units()[0]

    def getMeanEnergy(self):
        return self._units()[1]

    def getConvEnergy(self):
        return self._units()[2]

    def getConvLength(self):
        return self._units()[3]

    def _settings(self):
        out = []
        if self._settings_file is None:
            return out
        with open(self._settings_file) as fh:
            for line in fh:
                w = line.split("#", 1)[0].split()
                if w:
                    out.append((w[0], " ".join(w[1:])))
        return out

    def settingsKeywordExists(self, keyword):
        return any(k == keyword for k, _ in self._settings())

    def settingsGetValue(self, keyword):
        for k, v in self._settings():
            if k == keyword:
                return v
        raise KeyError(f'keyword "{keyword}" not found')

    # ---- energy offsets ----------------------------------------------------
    def _offset(self, s):
        return sum(c * self._m.atomic_energy_offset(e)
                   for e, c in enumerate(s.numAtomsPerElement))

    def addEnergyOffset(self, structure, ref=True):
        if ref:
            structure.energyRef += self._offset(structure)
        else:
            structure.energy += self._offset(structure)

    def removeEnergyOffset(self, structure, ref=True):
        if ref:
            structure.energyRef -= self._offset(structure)
        else:
            structure.energy -= self._offset(structure)

    # ---- evaluation steps --------------------------------------------------
    def calculateSymmetryFunctions(self, structure, derivatives):
        self.calculateSymmetryFunctionGroups(structure, derivatives)

    def calculateSymmetryFunctionGroups(self, structure, derivatives):
        s = structure
        rc = self.getMaxCutoffRadius()
        if s._cutoff is None:
            raise RuntimeError("ERROR: Neighbor list not calculated "
                               "(Structure.calculateNeighborList).\n")
        if s._cutoff < rc * (1.0 - 1e-12):
            raise ValueError(f"ERROR: Neighbor list cutoff {s._cutoff} is "
                             f"below the potential's {rc}.\n")
        r, box = s._physical_positions()
        self._m.set_structure(r, s._elem, box, remap=s.isPeriodic)
        self._m.calculate_neighbor_list()
        self._m.calculate_symmetry_function_groups(bool(derivatives))
        self._uploaded = s._token
        s._numNeighbors = self._m.neighbor_counts()
        s._numSF = [self._m.num_symmetry_functions(e)
                    for e in range(self._m.num_elements)]
        s._G = self._m.symmetry_functions()
        s._dEdG = None
        s.hasSymmetryFunctions = True
        s.hasSymmetryFunctionDerivatives = bool(derivatives)

    def _require(self, s):
        if self._uploaded is not s._token:
            raise RuntimeError("ERROR: Calculate the symmetry functions of "
                               "this structure first.\n")

    def calculateAtomicNeuralNetworks(self, structure, derivatives):
        s = structure
        self._require(s)
        self._m.calculate_atomic_neural_networks(bool(derivatives))
        _, ce = s._energy_scale()
        s._energyAtom[:] = self._m.atomic_energies() * ce
        if derivatives:
            # dE/dG arrives in normalized units (as held during evaluateNNP).
            d = self._m.dEdG()
            s._dEdG = d if s._norm is not None else d / self.getConvEnergy()

    def calculateEnergy(self, structure):
        s = structure
        self._require(s)
        self._m.calculate_energy()
        mean, ce = s._energy_scale()
        e = self._m.energy - self._offset(s)
        s.energy = (e - s.numAtoms * mean) * ce

    def calculateForces(self, structure):
        s = structure
        self._require(s)
        self._m.calculate_forces()
        f = self._m.forces()
        if s._norm is not None:
            f = f * (s._norm[1] / s._norm[2])
        s._f[:] = f

    def _evaluate(self, s, use_forces=True):
        """Mode::evaluateNNP (Mode.cpp:1967-2016) for a 2G potential."""
        s.calculateNeighborList(self.getMaxCutoffRadius())
        self.calculateSymmetryFunctionGroups(s, use_forces)
        self.calculateAtomicNeuralNetworks(s, True)
        self.calculateEnergy(s)
        if use_forces:
            self.calculateForces(s)

    def close(self):
        self._m.close()


class Prediction(Mode):
    """nnp::Prediction (src/pynnp/Prediction.pyx, libnnp/Prediction.cpp)."""

    def __init__(self, device: int = 0):
        super().__init__(device)
        self.fileNameSettings = "input.nn"
        self.fileNameScaling = "scaling.data"
        self.formatWeightsFilesShort = "weights.%03zu.data"
        self.formatWeightsFilesCharge = "weightse.%03zu.data"
        self.structure = Structure()

    def setup(self):
        """Prediction::setup (Prediction.cpp:34-46)."""
        self.initialize()
        self.loadSettingsFile(self.fileNameSettings)
        self.setupGeneric()
        self.setupSymmetryFunctionScaling(self.fileNameScaling)
        self.setupNeuralNetworkWeights(self.formatWeightsFilesShort)
        self.setupSymmetryFunctionStatistics(False, False, True, False)

    def readStructureFromFile(self, fileName="input.data"):
        """Prediction::readStructureFromFile (Prediction.cpp:48-63)."""
        s = self.structure
        s.reset()
        s.setElementMap(self.elementMap)
        s.readFromFile(fileName)
        self.removeEnergyOffset(s)
        norm, mean, ce, cl = self._units()
        if norm:
            s.toNormalizedUnits(mean, ce, cl)

    def predict(self):
        """Prediction::predict (Prediction.cpp:65-76)."""
        s = self.structure
        self._evaluate(s)
        norm, mean, ce, cl = self._units()
        if norm:
            s.toPhysicalUnits(mean, ce, cl)
        self.addEnergyOffset(s, False)
        self.addEnergyOffset(s, True)
