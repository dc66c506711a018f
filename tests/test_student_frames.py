"""Training frames of the student distillation (host only): isotropic strain
within the stated bound and Gaussian noise of the stated width, one width
for all frames or one drawn per frame from [sigma, sigma_max]."""
import numpy as np

from n2p2_b200 import student, synth


def _strain_and_noise(pos, x):
    s = float(np.sum(pos * x) / np.sum(pos * pos))   # least-squares scale
    return s, float(np.std(x - s * pos))


def test_fixed_width_frames():
    frames, elem = student.training_frames(6, sigma=0.15, strain=0.03,
                                           n_mol=512)
    _, pos, elem0 = synth.water_box(512, 2026)
    assert np.array_equal(elem, elem0)
    for box, x in frames:
        s, sd = _strain_and_noise(pos, x)
        assert abs(s - 1.0) <= 0.03 + 1e-3
        assert np.allclose(box, synth.water_box(512, 2026)[0] * s, rtol=1e-3)
        assert abs(sd - 0.15) < 0.01


def test_noise_width_range():
    frames, _ = student.training_frames(12, sigma=0.05, sigma_max=0.2,
                                        n_mol=512)
    _, pos, _ = synth.water_box(512, 2026)
    widths = [_strain_and_noise(pos, x)[1] for _, x in frames]
    assert min(widths) >= 0.05 - 0.005 and max(widths) <= 0.2 + 0.01
    assert max(widths) - min(widths) > 0.03      # widths differ per frame


def test_frames_are_reproducible():
    a, _ = student.training_frames(2, n_mol=64)
    b, _ = student.training_frames(2, n_mol=64)
    for (ba, xa), (bb, xb) in zip(a, b):
        assert np.array_equal(ba, bb) and np.array_equal(xa, xb)
