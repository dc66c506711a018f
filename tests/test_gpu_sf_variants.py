"""GPU parity of every symmetry-function kernel variant.

The autotuner may pick any launch variant of the symmetry-function stage
(per-owner kernels 0-5, staged-triplet kernels 6 and 7), so each one is
checked against the reference library on its own (N2P2B_SF_VARIANT forces
the variant of a new context).  Variants that do not fit a potential's
groups run the library's fallback for it; they are checked all the same.
Tolerances as in test_gpu_parity.py: G, dE/dG, dG/dr 1e-12 of the array's
scale; energy 1e-10 relative; forces |dF| <= 1e-10 max(|F|, rms F).  The
mixed form (FP32 symmetry functions) is checked against its accuracy
targets, E/atom RMSE <= 1e-4 and force RMSE <= 5e-3.
"""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials")
VARIANTS = list(range(8))


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _models(name, variant, monkeypatch, precision="fp64"):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    monkeypatch.setenv("N2P2B_SF_VARIANT", str(variant))
    d = os.path.join(POT, name)
    p = Prediction(d)
    p.setup()
    if precision != "fp64":
        p.set_precision(precision)
    return p, RefModel(d)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_variant_intermediates(gpu, monkeypatch, name, variant):
    _check_intermediates(*_models(name, variant, monkeypatch))


@pytest.mark.parametrize("variant", [6, 7])
@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_staged_batched_path(gpu, monkeypatch, name, variant):
    """The staged kernel's batched path (owners in batches, lanes over
    (member, partner slice)), which serves groups of four eta runs, forced
    for every narrow group by N2P2B_SF_LOCKSTEP=0."""
    monkeypatch.setenv("N2P2B_SF_LOCKSTEP", "0")
    _check_intermediates(*_models(name, variant, monkeypatch))


def _check_intermediates(p, ref):
    box, pos, elem = synth.water_box(64, 3)
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    G0, G1 = ref.G(), p.symmetry_functions()
    assert np.abs(G0 - G1).max() <= 1e-12 * max(1.0, np.abs(G0).max())
    D0, D1 = ref.dEdG(), p.dEdG()
    assert np.abs(D0 - D1).max() <= 1e-12 * np.abs(D0).max()
    cnt, idx, dr, d = ref.neighbors()
    S = max(ref.num_slots(e, f) for e in range(2) for f in range(2))
    s0 = ref.dGdr_self()
    n0 = ref.dGdr_nbr(len(idx), S)
    s1, n1 = p.dGdr()
    assert np.abs(s0 - s1).max() <= 1e-12 * np.abs(s0).max()
    assert np.abs(n0 - n1).max() <= 1e-12 * np.abs(n0).max()


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_variant_energy_forces(gpu, monkeypatch, name, variant):
    p, ref = _models(name, variant, monkeypatch)
    box, pos, elem = synth.water_box(512, 5)
    pos = pos + np.random.default_rng(5).normal(0.0, 0.1, pos.shape)
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    e1, f1 = p.predict(pos, elem, box)
    assert abs(e1 - e0) <= 1e-10 * abs(e0)
    scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    assert np.all(np.abs(f1 - f0) <= 1e-10 * scale)
    # Deterministic: a second evaluation reproduces every bit.
    e2, f2 = p.predict(pos, elem, box)
    assert e2 == e1 and np.array_equal(f2, f1)


@pytest.mark.parametrize("variant", [0, 4, 5, 6, 7])
@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_variant_mixed_accuracy(gpu, monkeypatch, name, variant):
    p, ref = _models(name, variant, monkeypatch, "mixed")
    box, pos, elem = synth.water_box(512, 9)
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    e1, f1 = p.predict(pos, elem, box)
    n = len(elem)
    assert abs(e1 - e0) / n <= 1e-4
    assert np.sqrt(np.mean((f1 - f0) ** 2)) <= 5e-3


def test_fp64_exponential(gpu):
    """The kernels' own FP64 exponential for x <= 0 (Cody-Waite reduction,
    Taylor polynomial) against libm (numpy) and CUDA's exp: within 2 ulp
    where the result is normal; below the smallest normal number (libm's
    subnormal range) it stays below that number too."""
    import ctypes
    from n2p2_b200 import _capi
    lib = _capi.load()
    rng = np.random.default_rng(3)
    x = np.concatenate([-rng.uniform(0.0, 1.0, 100000),
                        -rng.uniform(0.0, 50.0, 100000),
                        -rng.uniform(0.0, 750.0, 100000),
                        -np.array([0.0, 1e-300, 1e-17, 0.5 * np.log(2.0),
                                   np.log(2.0), 708.3, 708.4, 745.2, 800.0])])
    y = np.empty(2 * len(x))
    rc = lib.n2p2b_check_exp(x.ctypes.data_as(ctypes.c_void_p),
                             y.ctypes.data_as(ctypes.c_void_p), len(x))
    assert rc == 0
    ours, cuda = y[:len(x)], y[len(x):]
    ref = np.exp(x)
    normal = ref >= np.finfo(np.float64).tiny
    ulp = np.spacing(ref[normal])
    assert np.max(np.abs(ours[normal] - ref[normal]) / ulp) <= 2.0
    assert np.max(np.abs(ours[normal] - cuda[normal]) / ulp) <= 2.0
    assert np.all(np.abs(ours[~normal]) < np.finfo(np.float64).tiny)
