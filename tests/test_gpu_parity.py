"""GPU parity of the full prediction path against the reference library.

The oracle is the unmodified reference n2p2 compiled from its own sources
(oracle/_ref/libn2p2ref.so, pinned to the reference's golden vectors by
tests/test_oracle_golden.py).  Tolerances:
  * neighbor lists: bit-exact (same indices, same displacement bits, same
    distances) in the reference's list order;
  * symmetry functions, dE/dG, dG/dr: 1e-12 relative to the array's scale
    (FP64 with different summation order / libm);
  * energy: 1e-10 relative; forces: |dF| <= 1e-10 * max(|F|, rms(F)).
"""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials")


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _models(name):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    d = os.path.join(POT, name)
    p = Prediction(d)
    p.setup()
    return p, RefModel(d)


def _ref_entries(ref):
    cnt, idx, dr, d = ref.neighbors()
    return cnt, idx, dr, d


@pytest.mark.parametrize("nmol,seed", [(64, 7), (512, 11)])
def test_neighbor_list_bit_exact(gpu, nmol, seed):
    p, ref = _models("h2o_52")
    box, pos, elem = synth.water_box(nmol, seed)
    pos = pos + np.random.default_rng(seed).normal(0, 0.1, pos.shape)
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    p.set_structure(pos, elem, box)
    p.calculate_neighbor_list()
    c0, i0, dr0, d0 = _ref_entries(ref)
    c1, i1, dr1, d1 = p.neighbor_list()
    assert np.array_equal(c0, c1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(dr0.view(np.int64), dr1.view(np.int64))
    assert np.array_equal(d0.view(np.int64), d1.view(np.int64))


@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_intermediates_match(gpu, name):
    p, ref = _models(name)
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


@pytest.mark.parametrize("name,nmol", [("h2o_52", 64), ("h2o_52", 512),
                                       ("h2o_92", 64)])
def test_energy_forces(gpu, name, nmol):
    p, ref = _models(name)
    box, pos, elem = synth.water_box(nmol, 5)
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    e1, f1 = p.predict(pos, elem, box)
    assert abs(e1 - e0) <= 1e-10 * abs(e0)
    scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    assert np.all(np.abs(f1 - f0) <= 1e-10 * scale)
