"""GPU parity of the extrapolation-warning check
(Element::updateSymmetryFunctionStatistics) against the reference.

A compressed water box pushes symmetry functions outside the scaling.data
range; the number of warnings (symmetry functions outside [Gmin, Gmax] by
more than 1000 DBL_EPSILON) must equal the reference's count exactly, and the
per-atom counts must match the same test applied to the reference's G.
"""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials",
                   "h2o_52")


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scaling(path):
    """scaling.data rows: element, SF (1-based), min, max, mean, sigma."""
    rows = [ln.split() for ln in open(path)
            if ln.strip() and not ln.lstrip().startswith("#")]
    out = {}
    for r in rows:
        out[(int(r[0]) - 1, int(r[1]) - 1)] = tuple(float(x) for x in r[2:6])
    return out


def _compressed(factor, seed):
    box, pos, elem = synth.water_box(64, seed)
    return box * factor, pos * factor, elem


@pytest.mark.parametrize("factor", [0.92, 1.0])
def test_extrapolation_count_matches_reference(gpu, factor):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    box, pos, elem = _compressed(factor, 13)
    ref = RefModel(POT)
    ref.setup_statistics(collect_ew=True)
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    n_ref = ref.num_extrapolation_warnings()

    p = Prediction(POT)
    p.setup()
    p.setup_symmetry_function_statistics(False, True, False, False)
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    assert p.get_num_extrapolation_warnings() == n_ref
    counts = p.extrapolation_counts()
    assert counts.sum() == n_ref

    # The same test on the reference's G (center-only scaling: raw = G + mean).
    sc = _scaling(os.path.join(POT, "scaling.data"))
    G = ref.G()
    eps = 1000.0 * np.finfo(float).eps
    want = np.zeros(len(elem), dtype=np.int64)
    for i in range(len(elem)):
        e = int(elem[i])
        for s in range(ref.num_sf[e]):
            gmin, gmax, gmean, _ = sc[(e, s)]
            v = G[i, s] + gmean
            want[i] += (v + eps < gmin) or (v - eps > gmax)
    assert np.array_equal(counts, want)
    if factor < 1.0:
        assert n_ref > 0

    # Cumulative count and reset (Mode::getNumExtrapolationWarnings).
    p.evaluate_nnp(True)
    assert p.get_num_extrapolation_warnings() == 2 * n_ref
    p.reset_extrapolation_warnings()
    assert p.get_num_extrapolation_warnings() == 0


def test_extrapolation_write_and_stop(gpu, capfd):
    from n2p2_b200.mode import ExtrapolationError, Prediction
    box, pos, elem = _compressed(0.92, 13)
    p = Prediction(POT)
    p.setup()            # Prediction::setup writes warnings, like n2p2
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    err = capfd.readouterr().err
    assert "### NNP EXTRAPOLATION WARNING ### STRUCTURE:      0 ATOM:" in err
    p.setup_symmetry_function_statistics(False, False, False, True)
    with pytest.raises(ExtrapolationError):
        p.evaluate_nnp(True)
    # Results of the evaluation that raised are complete.
    e = p.energy
    assert np.isfinite(e)
