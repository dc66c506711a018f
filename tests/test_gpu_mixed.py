"""GPU accuracy of the mixed-precision form against the FP64 reference.

The mixed form computes symmetry functions and dG/dr in FP32 and the atomic
NNs on the tensor cores (BF16 operands, FP32 accumulation), with FP64
displacements, energy sum and force accumulation.  Its accuracy targets are
stated as root-mean-square errors against the double-precision reference:
  * energy per atom (total energy / atoms):  RMSE <= 1e-4 energy units;
  * force components:                        RMSE <= 5e-3 energy / length.
The intermediates are checked at looser, format-sized bounds that catch a
wrong operand layout (which produces errors of order one) long before the
end-to-end tolerances would.
"""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials")

E_PER_ATOM_RMSE = 1e-4
F_RMSE = 5e-3


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _pair(name, mode="mixed"):
    from n2p2_b200.mode import Prediction
    from oracle.ref import RefModel
    d = os.path.join(POT, name)
    p = Prediction(d)
    p.setup()
    p.set_precision(mode)
    return p, RefModel(d)


def _rel_rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


@pytest.mark.parametrize("mode", ["mixed", "bf16"])
@pytest.mark.parametrize("name", ["h2o_52", "h2o_92"])
def test_mixed_intermediates(gpu, name, mode):
    p, ref = _pair(name, mode)
    assert p.precision == mode
    box, pos, elem = synth.water_box(64, 3)
    ref.set_structure(pos, elem, box)
    ref.evaluate(True)
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    G0, G1 = ref.G(), p.symmetry_functions()
    # FP32 symmetry functions, relative to the scale of each SF column
    # (centered columns lose digits to the cancellation G - mean), with a
    # floor at 1e-3 of the largest column for the O-O radial functions of
    # large eta, which are ~1e-15 everywhere.
    scale = np.maximum(np.abs(G0).max(axis=0), 1e-3 * np.abs(G0).max())
    assert (np.abs(G1 - G0) / scale).max() < 5e-3
    s0 = ref.dGdr_self()
    s1, _ = p.dGdr()
    assert _rel_rms(s1, s0) < 1e-4
    # Tensor-core network: dE/dG and atomic energies within a few roundings
    # of the operand format (BF16: 2^-9; split: ~2^-17) of the FP64 values.
    tol = 5e-2 if mode == "bf16" else 1e-3
    D0, D1 = ref.dEdG(), p.dEdG()
    assert _rel_rms(D1, D0) < tol
    E0, E1 = ref.atomic_energies(), p.atomic_energies()
    assert _rel_rms(E1, E0) < tol


@pytest.mark.parametrize("mode", ["mixed", "bf16"])
@pytest.mark.parametrize("name,nmol,seed", [("h2o_52", 512, 5),
                                            ("h2o_92", 512, 6)])
def test_mixed_energy_force_rmse(gpu, name, nmol, seed, mode):
    """Both tensor-core forms meet the targets: hi/lo operands everywhere
    (mixed), or single BF16 deltas in the hidden layers' backward GEMMs
    (bf16)."""
    p, ref = _pair(name, mode)
    box, pos, elem = synth.water_box(nmol, seed)
    n = len(pos)
    rng = np.random.default_rng(seed)
    dE, dF = [], []
    for frame in range(3):
        x = pos + rng.normal(0.0, 0.1, pos.shape)
        ref.set_structure(x, elem, box)
        e0, f0 = ref.predict()
        e1, f1 = p.predict(x, elem, box)
        dE.append((e1 - e0) / n)
        dF.append((f1 - f0).ravel())
    e_rmse = float(np.sqrt(np.mean(np.square(dE))))
    f_rmse = float(np.sqrt(np.mean(np.square(np.concatenate(dF)))))
    print(f"{name} {mode}: energy/atom RMSE {e_rmse:.3e}, "
          f"force RMSE {f_rmse:.3e}")
    assert e_rmse <= E_PER_ATOM_RMSE
    assert f_rmse <= F_RMSE


def test_precision_switch_back_is_exact(gpu):
    """Switching back to FP64 restores the plain form's results exactly."""
    from n2p2_b200.mode import Prediction
    d = os.path.join(POT, "h2o_52")
    p = Prediction(d)
    p.setup()
    box, pos, elem = synth.water_box(64, 9)
    e0, f0 = p.predict(pos, elem, box)
    p.set_precision("mixed")
    p.predict(pos, elem, box)
    p.set_precision("fp64")
    e1, f1 = p.predict(pos, elem, box)
    assert e0 == e1
    assert np.array_equal(f0, f1)
