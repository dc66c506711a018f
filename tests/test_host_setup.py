"""Host-side setup of the library (C++, no GPU) against the reference.

A host-only context (device -1) parses input.nn / scaling.data / weights
exactly as Mode::setupGeneric + setupSymmetryFunctionScaling +
setupNeuralNetworkWeights do; its symmetry-function order (= NN input order
= scaling.data rows), parameters (normalized units), scaling factors and
dG/dr slot tables must equal the reference library's.
"""
import os

import numpy as np
import pytest

from conftest import REF_EXAMPLES
from oracle import ref as oref

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials")

needs_ref_lib = pytest.mark.skipif(not oref.ref_available(),
                                   reason="oracle/_ref not built")


def potential_dirs():
    out = [os.path.join(POT, d) for d in sorted(os.listdir(POT))
           if os.path.exists(os.path.join(POT, d, "input.nn"))]
    for name in ("H2O_RPBE-D3", "Cu2S_PBE", "Ethylbenzene_SCAN",
                 "DMABN_SCAN", "Anisole_SCAN"):
        out.append(os.path.join(REF_EXAMPLES, name))
    return out


def host_mode(d):
    from n2p2_b200.mode import Prediction
    p = Prediction(d, device=-1)
    p.setup()
    return p


@needs_ref_lib
@pytest.mark.parametrize("d", potential_dirs(),
                         ids=lambda d: os.path.basename(d))
def test_symmetry_function_setup_matches_reference(d):
    p = host_mode(d)
    r = oref.RefModel(d)
    assert p.num_elements == r.num_elements
    assert p.get_max_cutoff_radius() == r.max_cutoff
    for e in range(r.num_elements):
        assert p.num_symmetry_functions(e) == r.num_sf[e]
        for ne in range(r.num_elements):
            assert p.num_slots(e, ne) == r.num_slots(e, ne)
        for s in range(r.num_sf[e]):
            a = p.symmetry_function_params(e, s)
            b = r.sf_params(e, s)
            # type, e1, e2, eta, rs, rc, zeta, lambda, scaling, line: exact
            assert np.array_equal(a[:9], b[:9]), (e, s, a, b)
            assert a[9] == b[9]


@pytest.mark.parametrize("d", potential_dirs(),
                         ids=lambda d: os.path.basename(d))
def test_groups_partition_and_order(d):
    """Groups partition the SFs; members are sorted with eta slowest
    (SymGrpExpAngn::sortMembers) and share type, rc and elements.  Compact
    groups (types 20-22, SymGrpCompRad / SymGrpCompAngn) share type and
    elements only; their members are sorted by subtype, rc, rl, angles."""
    p = host_mode(d)
    for e in range(p.num_elements):
        groups = p.symmetry_function_groups(e)
        seen = sorted(s for g in groups for s in g)
        assert seen == list(range(p.num_symmetry_functions(e)))
        for g in groups:
            prm = [p.symmetry_function_params(e, s) for s in g]
            base = prm[0]
            compact = base[0] >= 20
            for q in prm:
                assert q[0] == base[0]
                assert q[1] == base[1] and q[2] == base[2]
                if not compact:
                    assert q[5] == base[5]
            idx = [4, 5, 3, 6, 7] if compact else [3, 4, 6, 7]
            keys = [tuple(q[idx]) for q in prm]
            assert keys == sorted(keys)


def test_missing_files_raise():
    from n2p2_b200.mode import Prediction
    p = Prediction("/nonexistent/dir", device=-1)
    with pytest.raises(Exception, match="Could not open"):
        p.setup()


def test_bad_settings_raise(tmp_path):
    from n2p2_b200.mode import Prediction
    (tmp_path / "input.nn").write_text(
        "number_of_elements 2\nelements H O\ncutoff_type 1\n"
        "mean_energy 1.0\n")  # incomplete normalization keywords
    p = Prediction(str(tmp_path), device=-1)
    with pytest.raises(Exception, match="normalization"):
        p.setup()


def test_evaluation_needs_a_device():
    from n2p2_b200.mode import Prediction, StateError
    p = host_mode(os.path.join(POT, "h2o_52"))
    with pytest.raises(StateError):
        p.set_structure(np.zeros((3, 3)), [1, 0, 0], None)
