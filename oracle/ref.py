"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes access to two CPU checkers of the n2p2 prediction path:

* ``RefModel`` drives the UNMODIFIED reference library compiled from the
  reference sources by ``oracle/Makefile`` (``oracle/_ref/libn2p2ref.so``,
  harness ``oracle/ref_harness.cpp``).  It follows ``Prediction::setup`` /
  ``readStructureFromFile`` / ``predict`` (libnnp/Prediction.cpp:34-76).
* ``read_input_data`` parses the reference's ``input.data`` format
  (libnnp/Structure.cpp:142-271) for test fixtures.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libn2p2ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_llp = C.POINTER(C.c_longlong)
_lib = None


def _p(a, ct):
    return a.ctypes.data_as(ct)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(REF_LIB):
        raise FileNotFoundError(
            f"{REF_LIB} missing: build it with `make -C oracle ref` "
            "(needs the reference sources)")
    L = C.CDLL(REF_LIB)
    L.refh_create.restype = C.c_void_p
    L.refh_create.argtypes = [C.c_char_p, C.c_int]
    L.refh_destroy.argtypes = [C.c_void_p]
    for f in ("refh_num_elements", "refh_num_atoms", "refh_max_threads"):
        getattr(L, f).restype = C.c_int
    L.refh_num_elements.argtypes = [C.c_void_p]
    L.refh_num_atoms.argtypes = [C.c_void_p]
    L.refh_max_threads.argtypes = []
    L.refh_num_sf.restype = C.c_int
    L.refh_num_sf.argtypes = [C.c_void_p, C.c_int]
    L.refh_num_slots.restype = C.c_int
    L.refh_num_slots.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.refh_max_cutoff.restype = C.c_double
    L.refh_max_cutoff.argtypes = [C.c_void_p]
    L.refh_sf_params.restype = C.c_int
    L.refh_sf_params.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    L.refh_set_structure.restype = C.c_int
    L.refh_set_structure.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _ip]
    L.refh_evaluate.restype = C.c_int
    L.refh_evaluate.argtypes = [C.c_void_p, C.c_int]
    L.refh_to_physical.restype = C.c_int
    L.refh_to_physical.argtypes = [C.c_void_p]
    L.refh_energy.restype = C.c_double
    L.refh_energy.argtypes = [C.c_void_p]
    for f in ("refh_positions", "refh_forces", "refh_atomic_energies"):
        getattr(L, f).argtypes = [C.c_void_p, _dp]
    L.refh_neighbor_counts.argtypes = [C.c_void_p, _llp]
    L.refh_neighbors.argtypes = [C.c_void_p, _llp, _dp, _dp]
    for f in ("refh_G", "refh_dEdG", "refh_dGdr_self", "refh_dGdr_nbr"):
        getattr(L, f).argtypes = [C.c_void_p, _dp, C.c_int]
    L.refh_time_stages.restype = C.c_int
    L.refh_time_stages.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    L.refh_setup_statistics.restype = C.c_int
    L.refh_setup_statistics.argtypes = [C.c_void_p] + [C.c_int] * 4
    L.refh_num_extrapolation_warnings.restype = C.c_long
    L.refh_num_extrapolation_warnings.argtypes = [C.c_void_p]
    L.refh_reset_extrapolation_warnings.argtypes = [C.c_void_p]
    _lib = L
    return L


class RefModel:
    """One reference ``Prediction`` set up from a potential directory.

    ``unscaled=True`` follows ``Mode::setupSymmetryFunctionScalingNone``
    instead of reading scaling.data (used to generate scaling statistics).
    """

    def __init__(self, directory: str, unscaled: bool = False):
        self.L = _load()
        self.h = self.L.refh_create(directory.encode(), int(unscaled))
        if not self.h:
            raise RuntimeError(f"reference setup failed for {directory}")
        self.num_elements = self.L.refh_num_elements(self.h)
        self.num_sf = [self.L.refh_num_sf(self.h, e)
                       for e in range(self.num_elements)]
        self.max_cutoff = self.L.refh_max_cutoff(self.h)
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.refh_destroy(self.h)
            self.h = None

    def num_slots(self, e: int, ne: int) -> int:
        return self.L.refh_num_slots(self.h, e, ne)

    def sf_params(self, e: int, s: int):
        """type, e1, e2, eta, rs, rc, zeta, lambda, scaling factor, line."""
        out = np.zeros(10)
        if self.L.refh_sf_params(self.h, e, s, _p(out, _dp)) != 0:
            raise RuntimeError("unknown symmetry function type")
        return out

    def set_structure(self, pos, elem, box=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        bp = None
        if box is not None:
            box = np.ascontiguousarray(box, dtype=np.float64).reshape(3, 3)
            bp = _p(box, _dp)
        if self.L.refh_set_structure(self.h, len(pos), bp, _p(pos, _dp),
                                     _p(elem, _ip)) != 0:
            raise RuntimeError("reference rejected the structure")
        self.n = len(pos)
        self.elem = elem.copy()

    def evaluate(self, forces: bool = True):
        """Mode::evaluateNNP in normalized units (intermediates comparable)."""
        if self.L.refh_evaluate(self.h, int(forces)) != 0:
            raise RuntimeError("reference evaluation failed")

    def predict(self):
        """Prediction::predict: evaluate + physical units + energy offsets."""
        self.evaluate(True)
        self.L.refh_to_physical(self.h)
        return self.energy(), self.forces()

    def energy(self) -> float:
        return self.L.refh_energy(self.h)

    def positions(self):
        out = np.zeros((self.n, 3))
        self.L.refh_positions(self.h, _p(out, _dp))
        return out

    def forces(self):
        out = np.zeros((self.n, 3))
        self.L.refh_forces(self.h, _p(out, _dp))
        return out

    def atomic_energies(self):
        out = np.zeros(self.n)
        self.L.refh_atomic_energies(self.h, _p(out, _dp))
        return out

    def neighbors(self):
        """(counts[N], index[E], dr[E,3], d[E]) in the reference's order."""
        cnt = np.zeros(self.n, dtype=np.int64)
        self.L.refh_neighbor_counts(self.h, _p(cnt, _llp))
        E = int(cnt.sum())
        idx = np.zeros(E, dtype=np.int64)
        dr = np.zeros((E, 3))
        d = np.zeros(E)
        self.L.refh_neighbors(self.h, _p(idx, _llp), _p(dr, _dp), _p(d, _dp))
        return cnt, idx, dr, d

    def G(self):
        s = max(self.num_sf)
        out = np.zeros((self.n, s))
        self.L.refh_G(self.h, _p(out, _dp), s)
        return out

    def dEdG(self):
        s = max(self.num_sf)
        out = np.zeros((self.n, s))
        self.L.refh_dEdG(self.h, _p(out, _dp), s)
        return out

    def dGdr_self(self):
        s = max(self.num_sf)
        out = np.zeros((self.n, s, 3))
        self.L.refh_dGdr_self(self.h, _p(out, _dp), s)
        return out

    def dGdr_nbr(self, num_entries: int, max_slots: int):
        out = np.zeros((num_entries, max_slots, 3))
        self.L.refh_dGdr_nbr(self.h, _p(out, _dp), max_slots)
        return out

    def setup_statistics(self, collect_statistics=False, collect_ew=False,
                         write_ew=False, stop_on_ew=False):
        """Mode::setupSymmetryFunctionStatistics (Prediction::setup turns
        on writing extrapolation warnings)."""
        self.L.refh_setup_statistics(self.h, int(collect_statistics),
                                     int(collect_ew), int(write_ew),
                                     int(stop_on_ew))

    def num_extrapolation_warnings(self) -> int:
        return int(self.L.refh_num_extrapolation_warnings(self.h))

    def reset_extrapolation_warnings(self):
        self.L.refh_reset_extrapolation_warnings(self.h)

    def time_stages(self, threads: int = 0, reps: int = 1):
        t = np.zeros(5)
        if self.L.refh_time_stages(self.h, threads, reps, _p(t, _dp)) != 0:
            raise RuntimeError("reference timing failed")
        return t


def max_threads() -> int:
    return _load().refh_max_threads()


def read_input_data(path: str):
    """Frames of an input.data file as dicts (box or None, pos, symbols).

    Follows the keyword layout read by Structure::readFromLines
    (libnnp/Structure.cpp:142-271): ``lattice`` rows, ``atom x y z El ...``.
    """
    frames = []
    cur = None
    with open(path) as fh:
        for line in fh:
            w = line.split()
            if not w:
                continue
            if w[0] == "begin":
                cur = {"box": [], "pos": [], "sym": [], "energy": 0.0}
            elif w[0] == "lattice":
                cur["box"].append([float(x) for x in w[1:4]])
            elif w[0] == "atom":
                cur["pos"].append([float(x) for x in w[1:4]])
                cur["sym"].append(w[4])
            elif w[0] == "energy":
                cur["energy"] = float(w[1])
            elif w[0] == "end":
                cur["box"] = (np.array(cur["box"]) if cur["box"] else None)
                cur["pos"] = np.array(cur["pos"])
                frames.append(cur)
                cur = None
    return frames


def read_golden_prediction(header_path: str):
    """Golden energies/forces from the reference's test/cpp/ExamplePrediction.h.

    Parsed at test time from the reference tree (never copied here):
    returns {example name: (energy, forces[N,3])}.
    """
    import re
    out = {}
    name = None
    energy = None
    forces = []
    num = r"([-+0-9.eE]+)"
    with open(header_path) as fh:
        for line in fh:
            m = re.search(r'ExamplePrediction\("([^"]+)"\)', line)
            if m:
                if name is not None:
                    out[name] = (energy, np.array(forces))
                name, energy, forces = m.group(1), None, []
                continue
            m = re.search(r"e->energy\s*=\s*" + num + ";", line)
            if m:
                energy = float(m.group(1))
                continue
            m = re.search(r"Vec3D\(\s*" + num + r",\s*" + num + r",\s*" + num
                          + r"\)", line)
            if m and "forces" in line:
                forces.append([float(m.group(k)) for k in (1, 2, 3)])
    if name is not None:
        out[name] = (energy, np.array(forces))
    return out
