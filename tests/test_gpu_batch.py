"""GPU tests of the batching form: many independent periodic structures
evaluated together must give, structure by structure, the reference's
neighbor lists (bit-exact), energies (1e-10 relative) and forces
(|dF| <= 1e-10 max(|F|, rms F)); a captured CUDA graph of the evaluation must
reproduce the direct evaluation bit for bit; the autotuner must keep the
results."""
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


def _pred():
    from n2p2_b200.mode import Prediction
    p = Prediction(POT)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    return p


def _noisy(structs, seed):
    rng = np.random.default_rng(seed)
    return [(b, x + rng.normal(0, 0.1, x.shape), e) for b, x, e in structs]


def _check_against_reference(p, structs):
    """Per structure: neighbor list bit-exact, energy 1e-10 relative, forces
    1e-10 max(|F|, rms F).  Returns the largest relative energy and force
    errors over the structures."""
    from oracle.ref import RefModel
    ref = RefModel(POT)
    ref.setup_statistics()
    worst_e = worst_f = 0.0
    E = p.structure_energies()
    F = p.forces()
    cnt, idx, dr, d = p.neighbor_list()
    a0 = e0 = 0
    for s, (box, x, el) in enumerate(structs):
        n = len(el)
        ref.set_structure(x, el, box)
        ref.evaluate(True)
        c_ref, i_ref, dr_ref, d_ref = ref.neighbors()
        m = int(c_ref.sum())
        assert np.array_equal(cnt[a0:a0 + n], c_ref)
        assert np.array_equal(idx[e0:e0 + m] - a0, i_ref)
        assert np.array_equal(dr[e0:e0 + m].view(np.int64),
                              dr_ref.view(np.int64))
        assert np.array_equal(d[e0:e0 + m].view(np.int64),
                              d_ref.view(np.int64))
        er, fr = ref.predict()
        assert abs(E[s] - er) <= 1e-10 * abs(er)
        f = F[a0:a0 + n]
        scale = np.maximum(np.abs(fr), np.sqrt(np.mean(fr ** 2)))
        assert np.all(np.abs(f - fr) <= 1e-10 * scale)
        worst_e = max(worst_e, abs(E[s] - er) / abs(er))
        worst_f = max(worst_f, float((np.abs(f - fr) / scale).max()))
        a0 += n
        e0 += m
    return worst_e, worst_f


def test_batch_matches_reference_per_structure(gpu):
    structs = _noisy(synth.batch_structures(7, 5, lo=11, hi=48), 1)
    p = _pred()
    p.set_structures(structs)
    p.evaluate_nnp(True)
    _check_against_reference(p, structs)
    assert abs(p.energy - p.structure_energies().sum()) <= 1e-12 * abs(
        p.energy)


def test_batch_full_size_range(gpu):
    """The batching workload's whole size range, 11-171 molecules (33-513
    atoms): 38 structures drawn from it plus one of each extreme size, in
    one batch, each against the reference alone."""
    structs = synth.batch_structures(38, 2029, lo=11, hi=171)
    for nmol, seed in ((11, 71), (171, 72)):
        structs.append(synth.water_box(nmol, seed))
    structs = _noisy(structs, 3)
    sizes = [len(s[2]) for s in structs]
    assert min(sizes) == 33 and max(sizes) == 513
    p = _pred()
    p.set_structures(structs)
    p.evaluate_nnp(True)
    we, wf = _check_against_reference(p, structs)
    print(f"{len(structs)} structures of {min(sizes)}-{max(sizes)} atoms: "
          f"max relative energy error {we:.1e}, force {wf:.1e}")


def test_graph_replay_equals_direct_evaluation(gpu):
    torch = gpu
    structs = synth.batch_structures(5, 9, lo=11, hi=40)
    frames = [_noisy(structs, k) for k in range(3)]
    p = _pred()
    p.set_structures(frames[0])
    p.evaluate_nnp(True)
    p.capture_graph(True)
    for fr in frames[1:]:
        x = np.concatenate([s[1] for s in fr])
        p.set_positions(torch.tensor(x, device="cuda"))
        p.launch_graph()
        p.finish()
        e_graph, f_graph = p.structure_energies(), p.forces()
        p.set_positions(x)
        p.evaluate_nnp(True)
        assert np.array_equal(e_graph, p.structure_energies())
        assert np.array_equal(f_graph, p.forces())


def test_single_structure_graph(gpu):
    box, pos, elem = synth.water_box(64, 4)
    p = _pred()
    p.set_structure(pos, elem, box)
    p.evaluate_nnp(True)
    p.capture_graph(True)
    x = pos + np.random.default_rng(0).normal(0, 0.1, pos.shape)
    p.set_positions(x)
    p.launch_graph()
    p.finish()
    e_graph, f_graph = p.energy, p.forces()
    p.evaluate_nnp(True)
    assert e_graph == p.energy
    assert np.array_equal(f_graph, p.forces())


def test_autotune_keeps_results(gpu):
    structs = _noisy(synth.batch_structures(6, 13, lo=11, hi=40), 2)
    p = _pred()
    p.set_structures(structs)
    p.evaluate_nnp(True)
    rep = p.autotune(True, 1)
    assert rep.startswith("bucket ")
    p.evaluate_nnp(True)
    _check_against_reference(p, structs)
