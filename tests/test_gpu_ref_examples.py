"""The reference's own regression examples through the GPU FP64 path.

The five nnp-predict examples of the reference's Prediction regression test
(test/cpp/ExamplePrediction.h, test/cpp/test_Prediction.cpp), committed with
their golden energies and forces under tests/golden/ref_examples:

  H2O_RPBE-D3        1,080 atoms; SF types 2 (r_s > 0) and 3; TANHU cutoff;
                     SCALECENTER; tanh; unit normalization
  Cu2S_PBE           144 atoms, monoclinic cell; SF types 2, 3 and 9; POLY2;
                     SCALESIGMA; softplus
  Ethylbenzene_SCAN  288 atoms; compact SF types 20 and 22; POLY2; softplus
  Anisole_SCAN       256 atoms, three elements; compact types
  DMABN_SCAN         21 atoms, no cell (non-periodic); three elements

Each runs through Prediction (setup, structure, predict: physical units and
atomic energy offsets) on the GPU and is checked
  * against the golden values at the reference's own tolerance,
    1000 * DBL_EPSILON (test_Prediction.cpp:27): forces absolutely, the
    energy relative to max(1, |E|) (the golden energies are sums of up to
    1,080 atomic energies, whose summation order differs here);
  * against the reference library on the same machine: neighbor lists
    bit-exact, energy 1e-10 relative, forces 1e-10 * max(|F|, rms F).
"""
import numpy as np
import pytest

from conftest import ref_example

pytestmark = pytest.mark.gpu

EXAMPLES = ["H2O_RPBE-D3", "Cu2S_PBE", "Ethylbenzene_SCAN", "Anisole_SCAN",
            "DMABN_SCAN"]
EPS1000 = 1000.0 * np.finfo(float).eps


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(name):
    from n2p2_b200.mode import Prediction
    d, box, pos, sym, ge, gf = ref_example(name)
    p = Prediction(d)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    elem = p.element_indices(sym)
    e, f = p.predict(pos, elem, box)
    return p, d, box, pos, elem, ge, gf, e, f


@pytest.mark.parametrize("name", EXAMPLES)
def test_example_golden(gpu, name):
    p, d, box, pos, elem, ge, gf, e, f = _run(name)
    de = abs(e - ge) / max(1.0, abs(ge))
    df = float(np.abs(f - gf).max())
    print(f"{name}: |dE|/max(1,|E|) = {de:.2e}, max |dF| = {df:.2e} "
          f"(1000 eps = {EPS1000:.2e})")
    p.close()
    assert de <= EPS1000
    assert df <= EPS1000


@pytest.mark.parametrize("name", EXAMPLES)
def test_example_vs_reference(gpu, name):
    from oracle.ref import RefModel
    p, d, box, pos, elem, ge, gf, e, f = _run(name)
    ref = RefModel(d)
    ref.setup_statistics()
    ref.set_structure(pos, elem, box)
    e0, f0 = ref.predict()
    ee = abs(e - e0) / abs(e0)
    scale = np.maximum(np.abs(f0), np.sqrt(np.mean(f0 ** 2)))
    ef = float((np.abs(f - f0) / scale).max())
    # neighbor lists in normalized units (what both evaluate on)
    ref.evaluate(True)
    c0, i0, dr0, d0 = ref.neighbors()
    c1, i1, dr1, d1 = p.neighbor_list()
    print(f"{name}: E {ee:.1e}, F {ef:.1e}, {len(i0)} neighbor entries")
    p.close()
    assert np.array_equal(c0, c1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(dr0.view(np.int64), dr1.view(np.int64))
    assert np.array_equal(d0.view(np.int64), d1.view(np.int64))
    assert ee <= 1e-10
    assert ef <= 1e-10
