"""GPU parity of the plain FP64 path across the settings the reference
supports, one axis at a time, against the reference library.

Every case writes a small two-element potential (H, O) into a temporary
directory -- radial type 2 with r_s = 0 and r_s > 0, narrow angular type 3
(also with r_s > 0), wide angular type 9, two cutoff radii (6 and 8 bohr) --
with seeded Nguyen-Widrow weights and scaling statistics of the unscaled
symmetry functions computed by the reference itself
(Mode::setupSymmetryFunctionScalingNone) over three frames, then evaluates
one structure on the GPU and in the reference.  Axes:

* cutoff functions: all nine types (CutoffFunction.cpp:120-213,
  CoreFunction.h), inner-cutoff parameter alpha = 0.2;
* scaling: ST_NONE, ST_SCALE, ST_CENTER, ST_SCALECENTER, ST_SCALESIGMA
  (SymFnc.cpp:150-195; keywords as Mode.cpp:715-751);
* activations: every letter of NeuralNetwork.cpp:1082-1091
  (l t s p r g c S e h);
* structures: a cubic periodic box, a triclinic periodic cell, and an open
  (non-periodic) cluster (Structure.cpp:357-391).

Tolerances: neighbor lists bit-exact (indices, displacement and distance
bits, reference order); symmetry functions 1e-12 of each column's scale;
dE/dG and dG/dr 1e-10 of the array's scale; energy 1e-10 relative; forces
|dF| <= 1e-10 * max(|F|, rms F).
"""
import math
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

ELEMENTS = ("H", "O")
PAIRS = (("H", "H"), ("H", "O"), ("O", "O"))


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def sf_lines():
    out = []
    for ec in ELEMENTS:
        for e1 in ELEMENTS:
            for eta, rs, rc in ((0.01, 0.0, 8.0), (0.1, 0.0, 8.0),
                                (0.5, 0.0, 6.0), (0.5, 2.0, 8.0),
                                (1.0, 3.5, 6.0)):
                out.append(f"symfunction_short {ec} 2 {e1} {eta} {rs} {rc}")
        for e1, e2 in PAIRS:
            for zeta in (1.0, 4.0):
                for lam in (-1.0, 1.0):
                    out.append(f"symfunction_short {ec} 3 {e1} {e2} 0.02 "
                               f"{lam} {zeta} 8.0")
            out.append(f"symfunction_short {ec} 3 {e1} {e2} 0.05 1.0 2.0 "
                       f"6.0 1.5")
            for zeta in (1.0, 2.0):
                for lam in (-1.0, 1.0):
                    out.append(f"symfunction_short {ec} 9 {e1} {e2} 0.03 "
                               f"{lam} {zeta} 8.0")
            out.append(f"symfunction_short {ec} 9 {e1} {e2} 0.05 -1.0 1.0 "
                       f"6.0 1.0")
    return out


SCALING = {
    "none": [],
    "scale": ["scale_symmetry_functions", "scale_min_short 0.0",
              "scale_max_short 1.0"],
    "center": ["center_symmetry_functions"],
    "scalecenter": ["scale_symmetry_functions", "center_symmetry_functions",
                    "scale_min_short -1.0", "scale_max_short 1.0"],
    "scalesigma": ["scale_symmetry_functions_sigma", "scale_min_short 0.0",
                   "scale_max_short 1.0"],
}


def nguyen_widrow(layers, acts, rng):
    """Connections in NeuralNetwork::setConnections order
    (NeuralNetwork.cpp:147-169) after U[-1, 1] and the Nguyen-Widrow
    modification (NeuralNetwork.cpp:269-310)."""
    W, b = [], []
    for i in range(1, len(layers)):
        W.append(rng.uniform(-1.0, 1.0, size=(layers[i], layers[i - 1])))
        b.append(rng.uniform(-1.0, 1.0, size=layers[i]))
    for i in range(1, len(layers) - 1):
        beta = 0.7 * math.pow(layers[i], 1.0 / float(layers[i - 1]))
        for j in range(layers[i]):
            s = math.sqrt(float(np.sum(W[i - 1][j] ** 2)))
            W[i - 1][j] *= beta / s
            b[i - 1][j] *= beta
            if acts[i - 1] == "t":
                W[i - 1][j] *= 2.0
                b[i - 1][j] *= 2.0
    W[-1][0][0] *= 0.5
    conn = []
    for Wl, bl in zip(W, b):
        for jin in range(Wl.shape[1]):
            for k in range(Wl.shape[0]):
                conn.append(Wl[k, jin])
        conn.extend(bl.tolist())
    return np.array(conn)


def frames_for_scaling():
    out = []
    for seed in (301, 302, 303):
        box, pos, elem = synth.water_box(64, seed)
        out.append((box, pos, elem))
    return out


def write_potential(d, cutoff="1 0.2", scaling="scalecenter",
                    acts=("t", "t", "l"), nodes=(12, 10), seed=5):
    from oracle.ref import RefModel
    os.makedirs(d, exist_ok=True)
    lines = sf_lines()
    with open(os.path.join(d, "input.nn"), "w") as f:
        f.write("number_of_elements 2\nelements H O\n")
        f.write(f"cutoff_type {cutoff}\n")
        for kw in SCALING[scaling]:
            f.write(kw + "\n")
        f.write(f"global_hidden_layers_short {len(nodes)}\n")
        f.write("global_nodes_short " + " ".join(map(str, nodes)) + "\n")
        f.write("global_activation_short " + " ".join(acts) + "\n")
        for ln in lines:
            f.write(ln + "\n")
    nsf = len(lines) // 2
    for e, z in ((0, 1), (1, 8)):
        rng = np.random.default_rng(seed + e)
        c = nguyen_widrow([nsf] + list(nodes) + [1], acts, rng)
        with open(os.path.join(d, f"weights.{z:03d}.data"), "w") as f:
            for v in c:
                f.write(f"{v:24.16E}\n")
    ref = RefModel(d, unscaled=True)
    vals = [[] for _ in range(2)]
    for box, pos, elem in frames_for_scaling():
        ref.set_structure(pos, elem, box)
        ref.evaluate(False)
        G = ref.G()
        for e in range(2):
            vals[e].append(G[elem == e, :ref.num_sf[e]])
    del ref
    with open(os.path.join(d, "scaling.data"), "w") as f:
        f.write("# e_index sf_index sf_min sf_max sf_mean sf_sigma\n")
        for e in range(2):
            a = np.concatenate(vals[e], axis=0)
            for k in range(a.shape[1]):
                f.write(f"{e + 1:6d} {k + 1:6d} {a[:, k].min():24.16E} "
                        f"{a[:, k].max():24.16E} {a[:, k].mean():24.16E} "
                        f"{np.std(a[:, k], ddof=1):24.16E}\n")
    return d


def cubic(seed=11):
    box, pos, elem = synth.water_box(64, seed)
    pos = pos + np.random.default_rng(seed).normal(0.0, 0.1, pos.shape)
    return box, pos, elem


def triclinic(seed=12):
    """The oxygens of a cubic water box carried over in fractional
    coordinates into a sheared cell (rows a, b, c), hydrogens at their
    molecule's offsets; some atoms lie outside the cell (remapped)."""
    box, pos, elem = synth.water_box(64, seed)
    L = box[0, 0]
    cell = np.array([[L, 0.0, 0.0],
                     [0.31 * L, 0.95 * L, 0.0],
                     [-0.22 * L, 0.17 * L, 1.04 * L]])
    out = pos.copy()
    for m in range(len(pos) // 3):
        o = pos[3 * m]
        onew = (o / L) @ cell
        out[3 * m:3 * m + 3] = pos[3 * m:3 * m + 3] - o + onew
    out += np.random.default_rng(seed).normal(0.0, 0.05, out.shape)
    return cell, out, elem


def cluster(seed=13):
    """An open cluster: the molecules of a 40-molecule box without the
    box (no periodic images)."""
    box, pos, elem = synth.water_box(40, seed)
    return None, pos, elem


def compare(d, structure):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    box, pos, elem = structure
    ref = RefModel(d)
    ref.setup_statistics()
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    p = Prediction(d)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    # neighbor lists: bit-exact
    c0, i0, dr0, d0 = ref.neighbors()
    c1, i1, dr1, d1 = p.neighbor_list()
    assert np.array_equal(c0, c1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(dr0.view(np.int64), dr1.view(np.int64))
    assert np.array_equal(d0.view(np.int64), d1.view(np.int64))
    # intermediates
    G0, G1 = ref.G(), p.symmetry_functions()
    scale = np.maximum(np.abs(G0).max(axis=0), 1e-3 * np.abs(G0).max())
    eg = float((np.abs(G1 - G0) / scale).max())
    D0, D1 = ref.dEdG(), p.dEdG()
    ed = float(np.abs(D0 - D1).max() / max(np.abs(D0).max(), 1e-300))
    S = max(ref.num_slots(e, f) for e in range(2) for f in range(2))
    n0 = ref.dGdr_nbr(len(i0), S)
    s0 = ref.dGdr_self()
    s1, n1 = p.dGdr()
    es = float(np.abs(s0 - s1).max() / np.abs(s0).max())
    en = float(np.abs(n0 - n1).max() / np.abs(n0).max())
    # energy and forces (physical units, offsets)
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    e1, f1 = p.predict(pos, elem, box)
    ee = abs(e1 - e0) / abs(e0)
    fs = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    ef = float((np.abs(f1 - f0) / fs).max())
    print(f"{os.path.basename(d)}: G {eg:.1e} dEdG {ed:.1e} dGdr(self) "
          f"{es:.1e} dGdr {en:.1e} E {ee:.1e} F {ef:.1e} "
          f"({len(i0)} neighbor entries)")
    p.close()
    assert eg <= 1e-12
    assert ed <= 1e-10
    assert es <= 1e-10 and en <= 1e-10
    assert ee <= 1e-10
    assert ef <= 1e-10


@pytest.mark.parametrize("ctype", list(range(9)))
def test_cutoff_types(gpu, tmp_path, ctype):
    d = write_potential(str(tmp_path / f"cut{ctype}"), cutoff=f"{ctype} 0.2")
    compare(d, cubic())


@pytest.mark.parametrize("scaling", sorted(SCALING))
def test_scaling_types(gpu, tmp_path, scaling):
    d = write_potential(str(tmp_path / f"scal_{scaling}"), cutoff="1 0.0",
                        scaling=scaling)
    compare(d, cubic(21))


@pytest.mark.parametrize("acts", [("s", "p", "l"), ("r", "g", "l"),
                                  ("c", "S", "l"), ("e", "h", "l"),
                                  ("t", "p", "t")])
def test_activations(gpu, tmp_path, acts):
    d = write_potential(str(tmp_path / ("act_" + "".join(acts))),
                        cutoff="2", acts=acts)
    compare(d, cubic(31))


@pytest.mark.parametrize("name,make", [("triclinic", triclinic),
                                       ("cluster", cluster)])
@pytest.mark.parametrize("ctype", ["1 0.0", "6 0.1"])
def test_cells(gpu, tmp_path, name, make, ctype):
    d = write_potential(str(tmp_path / f"{name}_{ctype[0]}"), cutoff=ctype)
    compare(d, make())
