"""LAMMPS's pair_style hdnnp, compiled unchanged against this library, on
the GPU (tests/lammps_stub/_build/lammps_pair_hdnnp, built by
tests/test_lammps_dropin_cpu.py from the reference's pair_hdnnp.cpp, the
drop-in include/InterfaceLammps.h and a single-rank LAMMPS stand-in).

One periodic water box: the pair style's settings, coeff, init_style and
compute(eflag, vflag) run as LAMMPS runs them, with ghost atoms, a full
neighbor list and the reverse communication of ghost forces.  Energy,
forces and per-atom energies must match the reference library
(Prediction::predict) -- energy 1e-10 relative, forces 1e-10 max(|F|,
rms F), atomic energies 1e-10 of their largest magnitude -- in LAMMPS units
(E / cfenergy, F cflength / cfenergy), also with cflength, cfenergy != 1.
"""
import os
import subprocess

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
POT = os.path.join(ROOT, "tests", "golden", "potentials", "h2o_52")
EXE = os.path.join(ROOT, "tests", "lammps_stub", "_build",
                   "lammps_pair_hdnnp")
SYM = {0: "H", 1: "O"}


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.access(EXE, os.X_OK):
        pytest.skip("lammps_pair_hdnnp not built (needs the reference tree)")
    return torch


def _write(path, box, pos, elem):
    with open(path, "w") as f:
        f.write("begin\n")
        for v in box:
            f.write("lattice %24.16E %24.16E %24.16E\n" % tuple(v))
        for r, e in zip(pos, elem):
            f.write("atom %24.16E %24.16E %24.16E %2s 0 0 0 0 0\n"
                    % (r[0], r[1], r[2], SYM[int(e)]))
        f.write("energy 0\ncharge 0\nend\n")


@pytest.mark.parametrize("cf", [(1.0, 1.0), (0.52917721, 27.211386)])
def test_pair_hdnnp_unchanged_matches_reference(gpu, tmp_path, cf):
    from oracle.ref import RefModel
    box, pos, elem = synth.water_box(32, 19)
    pos = np.mod(pos + np.random.default_rng(6).normal(0, 0.1, pos.shape),
                 box[0, 0])
    _write(tmp_path / "input.data", box, pos, elem)
    cfl, cfe = cf
    r = subprocess.run([EXE, POT, str(tmp_path / "input.data"), repr(cfl),
                        repr(cfe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    kv = {ln.split()[0]: ln.split()[1:] for ln in lines if ln.strip()}
    assert kv["requests"] == ["1", "flags", "1"]        # one full list
    e = float(kv["energy"][0])
    f = np.array([[float(x) for x in ln.split()[2:5]] for ln in lines
                  if ln.startswith("force ")])
    ea = np.array([float(ln.split()[2]) for ln in lines
                   if ln.startswith("eatom ")])
    log = [ln for ln in lines if ln.startswith("log ")]
    assert any("n2p2_b200" in ln for ln in log)
    ref = RefModel(POT)
    ref.setup_statistics()
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    a0 = ref.atomic_energies()
    assert abs(e * cfe - e0) <= 1e-10 * abs(e0)
    fs = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    assert np.all(np.abs(f * cfe / cfl - f0) <= 1e-10 * fs)
    assert np.abs(ea * cfe - a0).max() <= 1e-10 * np.abs(a0).max()


def _warning_fields(line):
    """(structure, atom, element, symfunc, type, value, min, max) of a
    "### NNP EXTRAPOLATION WARNING ###" line."""
    t = line.split()
    k = {t[i].rstrip(":"): t[i + 1] for i in range(5, len(t) - 1, 2)}
    return (int(k["STRUCTURE"]), int(k["ATOM"]), k["ELEMENT"],
            int(k["SYMFUNC"]), int(k["TYPE"]), float(k["VALUE"]),
            k["MIN"], k["MAX"])


def test_pair_hdnnp_extrapolation_warnings(gpu, tmp_path):
    """showew: the pair style writes the interface's warning lines through
    the log (InterfaceLammps::writeExtrapolationWarnings), element by
    element, symmetry function by symmetry function, with the LAMMPS tags
    as atom field -- the lines the reference writes for the same
    configuration, its G tested against scaling.data's range.  The EW
    buffer (fill, clear, extract) carries the same records."""
    from oracle.ref import RefModel
    box, pos, elem = synth.water_box(32, 23)
    box, pos = box * 0.92, np.mod(pos * 0.92, box[0, 0] * 0.92)
    _write(tmp_path / "input.data", box, pos, elem)
    r = subprocess.run([EXE, POT, str(tmp_path / "input.data"), "1.0", "1.0",
                        "showew"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    got = [ln[4:] for ln in lines
           if ln.startswith("log ### NNP EXTRAPOLATION WARNING ###")]
    buf = [ln[6:] for ln in lines
           if ln.startswith("ewbuf ### NNP EXTRAPOLATION WARNING ###")]
    assert got and buf == got

    ref = RefModel(POT)
    ref.setup_statistics(collect_ew=True)
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    assert len(got) == ref.num_extrapolation_warnings()
    # The reference's records: per element, per symmetry function, per atom.
    rows = [ln.split() for ln in open(os.path.join(POT, "scaling.data"))
            if ln.strip() and not ln.lstrip().startswith("#")]
    sc = {(int(q[0]) - 1, int(q[1]) - 1): [float(x) for x in q[2:5]]
          for q in rows}
    G = ref.G()
    eps = 1000.0 * np.finfo(float).eps
    want = []
    for e in range(2):
        for s in range(ref.num_sf[e]):
            gmin, gmax, gmean = sc[(e, s)]
            for i in np.flatnonzero(elem == e):
                v = G[i, s] + gmean        # center-only scaling
                if v + eps < gmin or v - eps > gmax:
                    want.append((0, int(i) + 1, SYM[e], s + 1,
                                 int(ref.sf_params(e, s)[0]), v,
                                 ("%10.3E" % gmin).strip(),
                                 ("%10.3E" % gmax).strip()))
    have = [_warning_fields(ln) for ln in got]
    assert [w[:5] + w[6:] for w in have] == [w[:5] + w[6:] for w in want]
    for h, w in zip(have, want):
        assert abs(h[5] - w[5]) <= 5e-4 * abs(w[5])
