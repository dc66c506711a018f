"""GPU tests of the distilled student: training gradients against finite
differences of the loss, a decreasing loss, the write / read round trip of
the student directory, and the gate (student for atoms inside its training
range, the teacher's own network for the others)."""
import os

import numpy as np
import pytest

from n2p2_b200 import synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials",
                   "h2o_52")
HIDDEN = 8


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def setup(gpu, tmp_path_factory):
    """A 64-molecule frame, its FP64 teacher labels and a fresh student."""
    from n2p2_b200 import student
    torch = gpu
    d = str(tmp_path_factory.mktemp("student"))
    box, pos, elem = synth.water_box(64, 21)
    x = pos + np.random.default_rng(3).normal(0, 0.1, pos.shape)
    E, F = student.label_frames(POT, [(box, x)], elem)
    e0 = E[0].cpu().numpy()
    student.make_student_dir(POT, d, {"H": 52, "O": 52}, HIDDEN, seed=5,
                             energy_bias={"H": float(e0[elem == 0].mean()),
                                          "O": float(e0[elem == 1].mean())})
    return {"dir": d, "box": box, "x": x, "elem": elem, "E": E[0], "F": F[0],
            "torch": torch}


def _ctx(s, mode="mixed"):
    from n2p2_b200.mode import Prediction
    p = Prediction(POT)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_precision(mode)
    p.setup_student(s["dir"])
    p.set_structure(s["x"], s["elem"], s["box"])
    p.calculate_neighbor_list()
    p.calculate_symmetry_function_groups(True)
    return p


def _offsets(nin=52, H=HIDDEN, elements=2):
    """Blob layout per element: W1 (H x nin), W1^T, b1, W2 (1 x H), W2^T,
    b2."""
    out, o = [], 0
    for _ in range(elements):
        d = {"W1": o, "W1T": o + H * nin, "b1": o + 2 * H * nin,
             "W2": o + 2 * H * nin + H, "W2T": o + 2 * H * nin + 2 * H,
             "b2": o + 2 * H * nin + 3 * H}
        out.append(d)
        o += 2 * H * nin + 3 * H + 1
    return out


def test_gradient_matches_finite_differences(setup):
    torch = setup["torch"]
    p = _ctx(setup)
    n = len(setup["elem"])
    batch = torch.tensor(np.random.default_rng(1).choice(n, 100, False)
                         .astype(np.int32), device="cuda")
    w0 = p.student_weights()
    l0 = p.student_train_step(setup["E"], setup["F"], batch, lr=0.0,
                              want_loss=True)
    g = p.student_gradient()
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    off = _offsets()
    nin, H = 52, HIDDEN
    picks = []
    for e in range(2):
        o = off[e]
        picks += [("W1", o["W1"] + 3 * nin + 7, o["W1T"] + 7 * H + 3),
                  ("W1", o["W1"] + 1 * nin + 40, o["W1T"] + 40 * H + 1),
                  ("b1", o["b1"] + 2, None), ("W2", o["W2"] + 5, o["W2T"] + 5),
                  ("b2", o["b2"], None)]
    for name, k, kt in picks:
        h = 1e-3 * max(1.0, abs(w0[k]))
        ls = []
        for sgn in (1, -1):
            w = w0.copy()
            w[k] += sgn * h
            if kt is not None:
                w[kt] = w[k]
            p.set_student_weights(w)
            l = p.student_train_step(setup["E"], setup["F"], batch, lr=0.0,
                                     want_loss=True)
            ls.append(l[0] + l[1])
        fd = (ls[0] - ls[1]) / (2 * h)
        scale = max(abs(fd), abs(g[k]), 1e-3 * (l0[0] + l0[1]))
        assert abs(fd - g[k]) <= 3e-2 * scale, (name, k, fd, g[k])
    p.set_student_weights(w0)


def test_training_reduces_loss(setup):
    torch = setup["torch"]
    p = _ctx(setup)
    n = len(setup["elem"])
    rng = np.random.default_rng(2)
    first = last = None
    for it in range(60):
        b = torch.tensor(rng.permutation(n)[:128].astype(np.int32),
                         device="cuda")
        l = p.student_train_step(setup["E"], setup["F"], b, lr=3e-3,
                                 want_loss=True)
        if first is None:
            first = l[0] + l[1]
        last = l[0] + l[1]
    assert last < 0.7 * first


def test_gate_and_round_trip(setup, tmp_path):
    from n2p2_b200.mode import Prediction
    p = _ctx(setup)
    p.student_update_range(reset=True)
    p.student_update_range()
    out = str(tmp_path)
    for f in ("input.nn", "scaling.data"):
        with open(os.path.join(setup["dir"], f)) as a, \
                open(os.path.join(out, f), "w") as b:
            b.write(a.read())
    p.student_write(out)
    w = p.student_weights()
    q = Prediction(POT)
    q.setup()
    q.setup_symmetry_function_statistics(False, False, False, False)
    q.set_precision("mixed")
    q.setup_student(out)
    assert np.array_equal(q.student_weights(), w)

    box, x, elem = setup["box"], setup["x"], setup["elem"]
    # Inside the training range: the gate passes every atom to the student.
    q.set_student_mode("only")
    q.set_structure(x, elem, box)
    q.evaluate_nnp(True)
    e_only = q.atomic_energies()
    q.set_student_mode("gated")
    q.evaluate_nnp(True)
    assert q.student_gated_count() == 0
    assert np.array_equal(q.atomic_energies(), e_only)

    # A compressed box leaves the range: gated atoms take the teacher's
    # (tensor-core) atomic energies, the others keep the student's.
    xs, bs = x * 0.93, box * 0.93
    q.set_student_mode("off")
    q.set_structure(xs, elem, bs)
    q.evaluate_nnp(True)
    e_teacher = q.atomic_energies()
    q.set_student_mode("only")
    q.evaluate_nnp(True)
    e_student = q.atomic_energies()
    q.set_student_mode("gated")
    q.evaluate_nnp(True)
    e_gated = q.atomic_energies()
    k = q.student_gated_count()
    assert 0 < k <= len(elem)
    from_teacher = e_gated == e_teacher
    from_student = e_gated == e_student
    assert np.all(from_teacher | from_student)
    assert int(from_teacher.sum()) >= k
