"""Generates the synthetic water potentials used by the tests and the bench.

    python tests/golden/make_potentials.py

Writes tests/golden/potentials/<name>/{input.nn, weights.001.data,
weights.008.data, scaling.data} for

* h2o_52 -- 52 SFs per element (radial eta 0.001..1.5 per neighbor element;
  narrow angular eta {0.001, 0.01, 0.05}, zeta {1, 4}, lambda +-1 per
  element pair), cos cutoff rc = 12 bohr, NN 52-25-25-1 (tanh, tanh, linear);
* h2o_92 -- the wide form: radial eta extended by {2.5, 4.0}, zeta
  {1, 2, 4, 16}: 92 SFs, NN 92-64-64-64-1 (softplus x3, linear);
* h2o_poly -- the compact (polynomial / exp bump) family: types 20, 21 and
  22 over all subtypes (p1..p4, asymmetric "a", e), angular windows that
  wrap around 0 and 180 degrees, and a p2 -> p3 member boundary with equal
  (rl, rc), which exercises the reuse of the r_jk radial value in
  SymGrpCompAngn; plus a few types 2 and 3 so that the compact paths run
  beside the Gaussian ones.  48 SFs, NN 48-20-20-1 (tanh, tanh, linear);
* h2o_wtd -- the element-weighted families: Gaussian types 12 and 13
  (weights: atomic numbers) with rs = 0 and rs > 0 members, and compact
  types 23, 24 and 25, beside a few types 2 and 3.  29 SFs, NN 29-15-15-1
  (tanh, tanh, linear).

    python tests/golden/make_potentials.py [name ...]   # default: all

Weights: seeded U[-1, 1] for every connection, then the Nguyen-Widrow
modification of NeuralNetwork::modifyConnections(MS_NGUYENWIDROW)
(libnnp/NeuralNetwork.cpp:269-310), restated here, in the weight order of
NeuralNetwork::setConnections (:147-169).

scaling.data: min / max / mean / sigma (n-1 normalization, the quantities
libnnptrain/Dataset.cpp:1064-1080 writes) of the UNSCALED symmetry
functions over 10 seeded 64-molecule water boxes, computed by the reference
library itself (oracle/_ref, Mode::setupSymmetryFunctionScalingNone).
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from n2p2_b200 import synth  # noqa: E402
from oracle.ref import RefModel  # noqa: E402

OUT = os.path.join(HERE, "potentials")
ELEMENTS = ["H", "O"]


def sf_lines(radial_eta, ang_eta, zetas, rc=12.0):
    lines = []
    for ec in ELEMENTS:
        for e1 in ELEMENTS:
            for eta in radial_eta:
                lines.append(f"symfunction_short {ec} 2 {e1} {eta} 0.0 {rc}")
        for e1, e2 in (("H", "H"), ("H", "O"), ("O", "O")):
            for eta in ang_eta:
                for zeta in zetas:
                    for lam in (-1.0, 1.0):
                        lines.append(f"symfunction_short {ec} 3 {e1} {e2} "
                                     f"{eta} {lam} {zeta} {rc}")
    return lines


def poly_lines():
    lines = []
    pairs = (("H", "H"), ("H", "O"), ("O", "O"))
    for ec in ELEMENTS:
        for e1 in ELEMENTS:
            for st, rl, rc in (("p2", 0.0, 12.0), ("p3", 0.0, 8.0),
                               ("p2a", 1.0, 6.0), ("e", 0.0, 10.0),
                               ("p4", 2.0, 12.0), ("p1", 0.0, 5.0)):
                lines.append(f"symfunction_short {ec} 20 {e1} {rl} {rc} {st}")
            for eta in (0.01, 0.1):
                lines.append(f"symfunction_short {ec} 2 {e1} {eta} 0.0 12.0")
        for e1, e2 in pairs:
            for al, ar in ((0.0, 90.0), (45.0, 135.0), (90.0, 180.0),
                           (-30.0, 30.0), (150.0, 210.0)):
                lines.append(f"symfunction_short {ec} 21 {e1} {e2} 0.0 12.0 "
                             f"{al} {ar} p2")
            lines.append(f"symfunction_short {ec} 21 {e1} {e2} 0.0 12.0 "
                         f"0.0 180.0 p3")
            lines.append(f"symfunction_short {ec} 21 {e1} {e2} 0.0 8.0 "
                         f"0.0 120.0 e")
            lines.append(f"symfunction_short {ec} 22 {e1} {e2} 0.0 10.0 "
                         f"0.0 180.0 p2")
            lines.append(f"symfunction_short {ec} 22 {e1} {e2} 0.0 10.0 "
                         f"60.0 120.0 p2")
            lines.append(f"symfunction_short {ec} 22 {e1} {e2} 0.5 9.0 "
                         f"30.0 150.0 p2a")
        for lam in (-1.0, 1.0):
            lines.append(f"symfunction_short {ec} 3 H H 0.01 {lam} 1.0 12.0")
    return lines


def wtd_lines():
    lines = []
    for ec in ELEMENTS:
        for eta, rs in ((0.001, 0.0), (0.01, 0.0), (0.03, 0.0), (0.1, 0.0),
                        (0.3, 0.0), (0.5, 2.0)):
            lines.append(f"symfunction_short {ec} 12 {eta} {rs} 12.0")
        for eta in (0.001, 0.01):
            for zeta in (1.0, 4.0):
                for lam in (-1.0, 1.0):
                    lines.append(f"symfunction_short {ec} 13 {eta} 0.0 "
                                 f"{lam} {zeta} 12.0")
        lines.append(f"symfunction_short {ec} 13 0.02 1.0 1.0 2.0 12.0")
        for st, rl, rc in (("p2", 0.0, 12.0), ("p3a", 1.0, 7.0),
                           ("e", 0.0, 9.0)):
            lines.append(f"symfunction_short {ec} 23 {rl} {rc} {st}")
        for al, ar in ((0.0, 100.0), (80.0, 180.0), (-40.0, 40.0)):
            lines.append(f"symfunction_short {ec} 24 0.0 11.0 {al} {ar} p2")
        for al, ar in ((30.0, 150.0), (0.0, 180.0)):
            lines.append(f"symfunction_short {ec} 25 0.0 9.0 {al} {ar} p4")
        for e1 in ELEMENTS:
            for eta in (0.01, 0.1):
                lines.append(f"symfunction_short {ec} 2 {e1} {eta} 0.0 12.0")
        for lam in (-1.0, 1.0):
            lines.append(f"symfunction_short {ec} 3 H H 0.01 {lam} 1.0 12.0")
    return lines


def write_input_nn(d, nodes, acts, lines):
    with open(os.path.join(d, "input.nn"), "w") as f:
        f.write("# Synthetic water potential (generated by "
                "tests/golden/make_potentials.py)\n")
        f.write("number_of_elements 2\n")
        f.write("elements H O\n")
        f.write("cutoff_type 1 0.0\n")
        # Centering only (ST_CENTER).  With rs = 0 and eta up to 4 bohr^-2
        # the O-O radial functions stay between 1e-15 and 1e-39 in every
        # generated frame (O-O >= 4.7 bohr), so min/max or sigma scaling
        # would multiply them by up to 1e38 and make the potential
        # numerically meaningless.
        f.write("center_symmetry_functions\n")
        f.write(f"global_hidden_layers_short {len(nodes)}\n")
        f.write("global_nodes_short " + " ".join(map(str, nodes)) + "\n")
        f.write("global_activation_short " + " ".join(acts) + "\n")
        for ln in lines:
            f.write(ln + "\n")


def nguyen_widrow(layers, acts, rng):
    """Connections (setConnections order) after U[-1,1] + Nguyen-Widrow."""
    W = []
    b = []
    for i in range(1, len(layers)):
        W.append(rng.uniform(-1.0, 1.0, size=(layers[i], layers[i - 1])))
        b.append(rng.uniform(-1.0, 1.0, size=layers[i]))
    for i in range(1, len(layers) - 1):
        beta = 0.7 * math.pow(layers[i], 1.0 / float(layers[i - 1]))
        tanh = acts[i - 1] == "t"
        for j in range(layers[i]):
            s = math.sqrt(float(np.sum(W[i - 1][j] ** 2)))
            W[i - 1][j] *= beta / s
            b[i - 1][j] *= beta
            if tanh:
                W[i - 1][j] *= 2.0
                b[i - 1][j] *= 2.0
    # Output layer: only weights[0] of the single output neuron is scaled.
    W[-1][0][0] *= 0.5
    conn = []
    for Wl, bl in zip(W, b):
        for jin in range(Wl.shape[1]):
            for k in range(Wl.shape[0]):
                conn.append(Wl[k, jin])
        conn.extend(bl.tolist())
    return np.array(conn)


def write_weights(d, nsf, nodes, acts, seed):
    for e, z in ((0, 1), (1, 8)):
        rng = np.random.default_rng(seed + e)
        c = nguyen_widrow([nsf] + list(nodes) + [1], acts, rng)
        with open(os.path.join(d, f"weights.{z:03d}.data"), "w") as f:
            f.write("# Seeded U[-1,1] + Nguyen-Widrow; setConnections order\n")
            for v in c:
                f.write(f"{v:24.16E}\n")


def write_scaling(d, n_frames=10, n_mol=64):
    ref = RefModel(d, unscaled=True)
    ne = ref.num_elements
    vals = [[] for _ in range(ne)]
    for f in range(n_frames):
        box, pos, elem = synth.water_box(n_mol, seed=1000 + f)
        ref.set_structure(pos, elem, box)
        ref.evaluate(False)
        G = ref.G()
        for e in range(ne):
            vals[e].append(G[elem == e, :ref.num_sf[e]])
    with open(os.path.join(d, "scaling.data"), "w") as f:
        f.write("#" + "#" * 80 + "\n")
        f.write("# Symmetry function scaling data (unscaled SF statistics "
                f"over {n_frames} water boxes of {n_mol} molecules).\n")
        f.write("# e_index sf_index sf_min sf_max sf_mean sf_sigma\n")
        f.write("#" + "#" * 80 + "\n")
        for e in range(ne):
            a = np.concatenate(vals[e], axis=0)
            n = a.shape[0]
            s = a.sum(axis=0)
            s2 = (a * a).sum(axis=0)
            for k in range(a.shape[1]):
                mean = s[k] / n
                # Two-pass variance: the one-pass form of Dataset.cpp cancels
                # catastrophically for the narrow zeta = 16 functions.
                sigma = float(np.std(a[:, k], ddof=1))
                f.write(f"{e + 1:10d} {k + 1:10d} {a[:, k].min():24.16E} "
                        f"{a[:, k].max():24.16E} {mean:24.16E} "
                        f"{sigma:24.16E}\n")


def make(name, radial_eta, ang_eta, zetas, nodes, acts, seed, lines=None):
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    if lines is None:
        lines = sf_lines(radial_eta, ang_eta, zetas)
    write_input_nn(d, nodes, acts, lines)
    nsf = len(lines) // 2
    write_weights(d, nsf, nodes, acts, seed)
    write_scaling(d)
    print(f"{name}: {nsf} SFs per element -> {d}")


if __name__ == "__main__":
    want = set(sys.argv[1:]) or {"h2o_52", "h2o_92", "h2o_poly", "h2o_wtd"}
    base_eta = [0.001, 0.01, 0.03, 0.06, 0.15, 0.3, 0.6, 1.5]
    if "h2o_52" in want:
        make("h2o_52", base_eta, [0.001, 0.01, 0.05], [1.0, 4.0],
             [25, 25], ["t", "t", "l"], seed=52)
    if "h2o_92" in want:
        make("h2o_92", base_eta + [2.5, 4.0], [0.001, 0.01, 0.05],
             [1.0, 2.0, 4.0, 16.0], [64, 64, 64], ["p", "p", "p", "l"],
             seed=92)
    if "h2o_poly" in want:
        make("h2o_poly", None, None, None, [20, 20], ["t", "t", "l"],
             seed=48, lines=poly_lines())
    if "h2o_wtd" in want:
        make("h2o_wtd", None, None, None, [15, 15], ["t", "t", "l"],
             seed=21, lines=wtd_lines())
