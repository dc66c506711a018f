"""ORACLE / TEST INFRASTRUCTURE ONLY.

Python front end of the C restatement (oracle/hdnnp_oracle.c): an
independent reader of n2p2's input.nn / scaling.data / weights.%03zu.data
(restating Mode::setupGeneric, setupSymmetryFunctionScaling and
readNeuralNetworkWeights, libnnp/Mode.cpp:212-2289) that fills the C
potential description, plus `predict()`.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libhdnnp_oracle.so")
MAXE = 8
MAXL = 8

_SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co "
    "Ni Cu Zn Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb "
    "Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re "
    "Os Ir Pt Au Hg Tl Pb Bi Po At Rn").split()
_ACT = {"l": 0, "t": 1, "s": 2, "p": 3, "r": 4, "g": 5, "c": 6, "S": 7,
        "e": 8, "h": 9}


class HoSF(C.Structure):
    _fields_ = [("type", C.c_int), ("e1", C.c_int), ("e2", C.c_int),
                ("eta", C.c_double), ("rs", C.c_double), ("rc", C.c_double),
                ("zeta", C.c_double), ("lambda_", C.c_double),
                ("zetaInt", C.c_int), ("useIntegerPow", C.c_int),
                ("scalingType", C.c_int), ("Smin", C.c_double),
                ("Gmin", C.c_double), ("Gmean", C.c_double),
                ("scalingFactor", C.c_double), ("slot", C.c_int * MAXE)]


class HoPotential(C.Structure):
    _fields_ = [("numElements", C.c_int), ("cutoffType", C.c_int),
                ("cutoffAlpha", C.c_double), ("numSF", C.c_int * MAXE),
                ("sfs", C.POINTER(HoSF) * MAXE),
                ("numSlots", (C.c_int * MAXE) * MAXE),
                ("numLayers", C.c_int * MAXE),
                ("neurons", (C.c_int * MAXL) * MAXE),
                ("activation", (C.c_int * MAXL) * MAXE),
                ("connections", C.POINTER(C.c_double) * MAXE),
                ("normalizeNeurons", C.c_int), ("normalize", C.c_int),
                ("meanEnergy", C.c_double), ("convEnergy", C.c_double),
                ("convLength", C.c_double), ("atomEnergy", C.c_double * MAXE)]


def _settings(path):
    """Keyword -> list of value strings (Settings::parseLines)."""
    out = {}
    with open(path) as fh:
        for line in fh:
            line = line.split("#")[0].split("!")[0]
            w = line.split()
            if not w:
                continue
            out.setdefault(w[0], []).append(" ".join(w[1:]))
    return out


def _sf_key(s):
    """SymFnc*::operator< (libnnp/SymFncExpRad.cpp:55-76,
    SymFncExpAngn.cpp:51-78)."""
    if s["type"] == 2:
        return (s["type"], s["rc"], s["eta"], s["rs"], s["e1"])
    return (s["type"], s["rc"], s["eta"], s["rs"], s["zeta"], s["lambda"],
            s["e1"], s["e2"])


class Potential:
    """A parsed potential directory, owning the ctypes arrays."""

    def __init__(self, directory: str):
        st = _settings(os.path.join(directory, "input.nn"))
        syms = sorted(st["elements"][0].split(), key=_SYMBOLS.index)
        ne = len(syms)
        self.symbols = syms
        if int(st["number_of_elements"][0]) != ne:
            raise ValueError("inconsistent number of elements")
        norm = all(k in st for k in ("mean_energy", "conv_energy",
                                     "conv_length"))
        convL = float(st["conv_length"][0]) if norm else 1.0
        ct = st["cutoff_type"][0].split()
        self.cutoff_type = int(ct[0])
        self.cutoff_alpha = float(ct[1]) if len(ct) > 1 else 0.0
        sfs = [[] for _ in range(ne)]
        for v in st.get("symfunction_short", []):
            a = v.split()
            s = {"ec": syms.index(a[0]), "type": int(a[1]), "rs": 0.0,
                 "zeta": 0.0, "lambda": 0.0, "e2": -1}
            if s["type"] == 2:
                s.update(e1=syms.index(a[2]), eta=float(a[3]),
                         rs=float(a[4]), rc=float(a[5]))
            else:
                e1, e2 = syms.index(a[2]), syms.index(a[3])
                s.update(e1=min(e1, e2), e2=max(e1, e2), eta=float(a[4]),
                         **{"lambda": float(a[5])}, zeta=float(a[6]),
                         rc=float(a[7]))
                if len(a) > 8:
                    s["rs"] = float(a[8])
            if norm:  # SymFnc*::changeLengthUnit
                s["eta"] /= convL * convL
                s["rs"] *= convL
                s["rc"] *= convL
            sfs[s["ec"]].append(s)
        for e in range(ne):
            sfs[e].sort(key=_sf_key)
        # slot tables (Element::setupSymmetryFunctionMemory)
        slots = np.zeros((MAXE, MAXE), dtype=np.int32)
        for e in range(ne):
            for s in sfs[e]:
                s["slot"] = [-1] * MAXE
                for f in range(ne):
                    rel = (f == s["e1"]) if s["type"] == 2 else \
                          (f in (s["e1"], s["e2"]))
                    if rel:
                        s["slot"][f] = int(slots[e, f])
                        slots[e, f] += 1
        # scaling
        if ("scale_symmetry_functions" in st
                and "center_symmetry_functions" not in st):
            stype = 1
        elif ("scale_symmetry_functions" not in st
              and "center_symmetry_functions" in st):
            stype = 2
        elif "scale_symmetry_functions" in st:
            stype = 3
        elif "scale_symmetry_functions_sigma" in st:
            stype = 4
        else:
            stype = 0
        smin = float(st.get("scale_min_short", ["0.0"])[0]) \
            if stype in (1, 3, 4) else 0.0
        smax = float(st.get("scale_max_short", ["1.0"])[0]) \
            if stype in (1, 3, 4) else 0.0
        rows = []
        with open(os.path.join(directory, "scaling.data")) as fh:
            for line in fh:
                if not line.startswith("#"):
                    rows.append([float(x) for x in line.split()])
        r = 0
        for e in range(ne):
            for s in sfs[e]:
                row = rows[r]
                r += 1
                gmin, gmax, gmean = row[2], row[3], row[4]
                sig = row[5] if len(row) > 5 else 0.0
                if stype in (0, 2):
                    sf = 1.0
                elif stype in (1, 3):
                    sf = (smax - smin) / (gmax - gmin)
                else:
                    sf = (smax - smin) / sig
                s.update(stype=stype, Smin=smin, Gmin=gmin, Gmean=gmean,
                         sf=sf)
        # NN topology (global keywords only) and weights
        nh = int(st["global_hidden_layers_short"][0])
        nodes = [int(x) for x in st["global_nodes_short"][0].split()]
        acts = st["global_activation_short"][0].split()
        P = HoPotential()
        P.numElements = ne
        P.cutoffType = self.cutoff_type
        P.cutoffAlpha = self.cutoff_alpha
        P.normalizeNeurons = int("normalize_nodes" in st)
        P.normalize = int(norm)
        if norm:
            P.meanEnergy = float(st["mean_energy"][0])
            P.convEnergy = float(st["conv_energy"][0])
            P.convLength = convL
        else:
            P.convEnergy = P.convLength = 1.0
        for v in st.get("atom_energy", []):
            a = v.split()
            P.atomEnergy[syms.index(a[0])] = float(a[1])
        self._keep = []
        for e in range(ne):
            arr = (HoSF * len(sfs[e]))()
            for k, s in enumerate(sfs[e]):
                t = arr[k]
                t.type, t.e1, t.e2 = s["type"], s["e1"], s["e2"]
                t.eta, t.rs, t.rc = s["eta"], s["rs"], s["rc"]
                t.zeta, t.lambda_ = s["zeta"], s["lambda"]
                t.zetaInt = int(round(s["zeta"]))
                t.useIntegerPow = int(abs(s["zeta"] - t.zetaInt)
                                      <= np.finfo(float).tiny)
                t.scalingType, t.Smin = s["stype"], s["Smin"]
                t.Gmin, t.Gmean, t.scalingFactor = s["Gmin"], s["Gmean"], s["sf"]
                for f in range(MAXE):
                    t.slot[f] = s["slot"][f]
            self._keep.append(arr)
            P.sfs[e] = C.cast(arr, C.POINTER(HoSF))
            P.numSF[e] = len(sfs[e])
            for f in range(MAXE):
                P.numSlots[e][f] = int(slots[e, f])
            layers = [len(sfs[e])] + nodes + [1]
            P.numLayers[e] = nh + 2
            for l, w in enumerate(layers):
                P.neurons[e][l] = w
            P.activation[e][0] = 0
            for l, a in enumerate(acts):
                P.activation[e][l + 1] = _ACT[a]
            z = _SYMBOLS.index(syms[e]) + 1
            w = []
            with open(os.path.join(directory, f"weights.{z:03d}.data")) as fh:
                for line in fh:
                    if line.startswith("#") or not line.split():
                        continue
                    w.append(float(line.split()[0]))
            warr = np.ascontiguousarray(w, dtype=np.float64)
            self._keep.append(warr)
            P.connections[e] = warr.ctypes.data_as(C.POINTER(C.c_double))
        self.P = P
        self.num_sf = [len(x) for x in sfs]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} missing: `make -C oracle restated`")
        L = C.CDLL(LIB)
        L.ho_predict.restype = C.c_int
        L.ho_predict.argtypes = [C.POINTER(HoPotential), C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                 C.c_void_p, C.c_void_p]
        L.ho_last_num_entries.restype = C.c_long
        L.ho_last_neighbors.argtypes = [C.c_void_p] * 4
        L.ho_last_G.argtypes = [C.c_void_p, C.c_int]
        _lib = L
    return _lib


_cache: dict = {}


def predict(directory, pos, elem, box=None, atomic=False):
    """(energy, forces[, atomic energies]) of the restated path."""
    L = _load()
    pot = _cache.get(directory)
    if pot is None:
        pot = _cache[directory] = Potential(directory)
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    elem = np.ascontiguousarray(elem, dtype=np.int32)
    n = len(pos)
    f = np.zeros((n, 3))
    ea = np.zeros(n)
    e = C.c_double()
    bp = None
    if box is not None:
        b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
        bp = b.ctypes.data
    rc = L.ho_predict(C.byref(pot.P), n, bp, pos.ctypes.data, elem.ctypes.data,
                      C.byref(e), f.ctypes.data, ea.ctypes.data)
    if rc != 0:
        raise RuntimeError("restated oracle failed")
    return (e.value, f, ea) if atomic else (e.value, f)


def last_neighbors():
    L = _load()
    E = L.ho_last_num_entries()
    return E


def last_G(n, stride):
    L = _load()
    G = np.zeros((n, stride))
    L.ho_last_G(G.ctypes.data, stride)
    return G
