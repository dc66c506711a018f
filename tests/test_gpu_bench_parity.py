"""Parity at the benchmarked size: the 24,576-atom water box that bench.py
times (8,192 molecules, L = 118.26 bohr, seed 2026, the 52-SF potential
h2o_52), as built and as its first timed frame (sigma = 0.1 bohr Gaussian
noise, seed 2027), through the GPU FP64 path and the reference library
(Structure::calculateNeighborList, Structure.cpp:287-399; Mode::evaluateNNP,
Mode.cpp:1967-2016).

  * neighbor lists: bit-exact (2.6 M entries: indices, displacement and
    distance bits, in the reference's order);
  * energy: 1e-10 relative;
  * forces: |dF| <= 1e-10 * max(|F|, rms F), per component;
  * atomic energies: 1e-10 of their largest magnitude.
"""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials",
                   "h2o_52")
N_MOL, SEED, SIGMA = 8192, 2026, 0.1


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def frames():
    box, pos, elem = synth.water_box(N_MOL, SEED)
    _, noisy = synth.noisy_frames(pos, 1, SIGMA, seed=SEED + 1, box=box)
    return box, elem, {"built": pos, "noisy": noisy[0]}


@pytest.mark.parametrize("which", ["built", "noisy"])
def test_bench_frame_parity(gpu, frames, which):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    box, elem, fr = frames
    pos = fr[which]
    ref = RefModel(POT)
    ref.setup_statistics()
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    a0 = ref.atomic_energies()
    c0, i0, dr0, d0 = ref.neighbors()
    p = Prediction(POT)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    e1, f1 = p.predict(pos, elem, box)
    a1 = p.atomic_energies()
    c1, i1, dr1, d1 = p.neighbor_list()
    p.close()
    assert len(elem) == 3 * N_MOL
    assert np.array_equal(c0, c1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(dr0.view(np.int64), dr1.view(np.int64))
    assert np.array_equal(d0.view(np.int64), d1.view(np.int64))
    ee = abs(e1 - e0) / abs(e0)
    scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    ef = float((np.abs(f1 - f0) / scale).max())
    ea = float(np.abs(a1 - a0).max() / np.abs(a0).max())
    rel = float(np.linalg.norm(f1 - f0) / np.linalg.norm(f0))
    print(f"{which}: {len(i0)} entries bit-exact; E {ee:.1e}, F {ef:.1e} "
          f"(normwise {rel:.1e}), atomic E {ea:.1e}")
    assert ee <= 1e-10
    assert ef <= 1e-10
    assert ea <= 1e-10
