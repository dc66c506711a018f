"""Copies the reference's nnp-predict example potentials and structures into
this directory and writes their golden energies and forces.

    N2P2_REFERENCE=/path/to/n2p2 python tests/golden/ref_examples/make_ref_examples.py

For each example of the reference's regression test of Prediction
(test/cpp/ExamplePrediction.h, checked by test/cpp/test_Prediction.cpp at
1000 * DBL_EPSILON) this copies examples/nnp-predict/<name>/{input.nn,
scaling.data, weights.*.data, input.data} unchanged, and writes golden.txt:

    energy <E>
    <fx> <fy> <fz>          (one line per atom, input.data order)

with the values parsed from ExamplePrediction.h.  It also writes
cutoff_kats.txt, the known answers of test/cpp/test_CutoffFunction.cpp:

    rc <rc> alpha <alpha> r <r>
    <type> <f> <df>         (one line per cutoff type 0..8)  These are test fixtures
(data the reference's own tests hold), used by tests/test_oracle_golden.py
and tests/test_gpu_ref_examples.py so that neither needs the reference tree.

What the examples exercise:
  H2O_RPBE-D3        1,080 atoms, cubic box; SF types 2 (r_s > 0) and 3;
                     TANHU cutoff; SCALECENTER scaling; tanh network;
                     unit normalization (mean_energy, conv_energy,
                     conv_length).
  Cu2S_PBE           144 atoms, monoclinic cell; SF types 2, 3 and 9; POLY2
                     cutoff; SCALESIGMA scaling; softplus.
  Ethylbenzene_SCAN  288 atoms, periodic; compact SF types 20 and 22; POLY2;
                     SCALECENTER; softplus.
  Anisole_SCAN       256 atoms, periodic, three elements; compact types.
  DMABN_SCAN         21 atoms, NON-periodic (no lattice), three elements;
                     compact types.
"""
from __future__ import annotations

import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
EXAMPLES = ["H2O_RPBE-D3", "Cu2S_PBE", "Ethylbenzene_SCAN", "Anisole_SCAN",
            "DMABN_SCAN"]


def parse_golden(header_path: str):
    """{name: (energy, [[fx, fy, fz], ...])} from ExamplePrediction.h."""
    out = {}
    name, energy, forces = None, None, []
    num = r"([-+0-9.eE]+)"
    with open(header_path) as fh:
        for line in fh:
            m = re.search(r'ExamplePrediction\("([^"]+)"\)', line)
            if m:
                if name is not None:
                    out[name] = (energy, forces)
                name, energy, forces = m.group(1), None, []
                continue
            m = re.search(r"e->energy\s*=\s*" + num + ";", line)
            if m:
                energy = m.group(1)
                continue
            m = re.search(r"Vec3D\(\s*" + num + r",\s*" + num + r",\s*" + num
                          + r"\)", line)
            if m and "forces" in line:
                forces.append([m.group(k) for k in (1, 2, 3)])
    if name is not None:
        out[name] = (energy, forces)
    return out


def parse_cutoff_kats(src_path: str):
    """(rc, alpha, r, f[9], df[9]) as strings from test_CutoffFunction.cpp
    (test radius = frac * rc)."""
    src = open(src_path).read()
    rc = re.search(r"cutoffRadius\s*=\s*([0-9.eE+-]+);", src).group(1)
    alpha = re.search(r"cutoffParameter\s*=\s*([0-9.eE+-]+);",
                      src).group(1)
    frac = re.search(r"testRadius\s*=\s*([0-9.eE+-]+)\s*\*", src).group(1)

    def vec(name):
        body = re.search(r"vector<double> const " + name +
                         r"\s*=\s*\{(.*?)\}", src, re.S).group(1)
        return [x.strip() for x in body.replace("\n", " ").split(",")]
    return rc, alpha, repr(float(frac) * float(rc)), vec("f"), vec("df")


def main():
    ref = os.environ.get("N2P2_REFERENCE", "/root/reference")
    src_root = os.path.join(ref, "examples", "nnp-predict")
    golden = parse_golden(os.path.join(ref, "test", "cpp",
                                       "ExamplePrediction.h"))
    for name in EXAMPLES:
        src = os.path.join(src_root, name)
        dst = os.path.join(HERE, name)
        os.makedirs(dst, exist_ok=True)
        for f in sorted(os.listdir(src)):
            if f in ("input.nn", "scaling.data", "input.data") or (
                    f.startswith("weights.") and f.endswith(".data")):
                shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
        energy, forces = golden[name]
        with open(os.path.join(dst, "golden.txt"), "w") as fh:
            fh.write(f"energy {energy}\n")
            for f in forces:
                fh.write(" ".join(f) + "\n")
        print(f"{name}: {len(forces)} atoms -> {dst}")
    rc, alpha, r, f, df = parse_cutoff_kats(
        os.path.join(ref, "test", "cpp", "test_CutoffFunction.cpp"))
    with open(os.path.join(HERE, "cutoff_kats.txt"), "w") as fh:
        fh.write(f"rc {rc} alpha {alpha} r {r}\n")
        for t, (a, b) in enumerate(zip(f, df)):
            fh.write(f"{t} {a} {b}\n")


if __name__ == "__main__":
    sys.exit(main())
