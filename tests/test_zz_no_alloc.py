"""GPU tests of n2p2b_neighbor_list_noalloc, the neighbor list for callers
that cannot allocate device memory while they run (for example an MD engine
that reserves all GPU memory at start-up and hands the library fixed
buffers, or a real-time loop that cannot afford cudaMalloc's device-wide
synchronization).

The entry point is called through the C-ABI with buffers the test owns,
several times in a row (its static scratch is reused between the calls),
and each result must equal, bit for bit (the tolerance of every
neighbor-list test here):
  * the list that the regular entry point (n2p2b_calculate_neighbor_list)
    builds for the same positions, and
  * where every atom lies inside the cell, the reference library's own
    Structure::calculateNeighborList (the oracle).
The cases reach each of its paths: the cell path with 3 or more cells per
axis, with one cell and with two (where the 27-cell stencil wraps onto the
same cells under different images), a skewed (triclinic) cell, the brute
path for a box smaller than the cutoff (several images per axis), for an
open structure (no box) and for an atom outside the cell; and a capacity one
entry short, which must fail with N2P2B_ERR_CAPACITY and report the
required size in *total.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from n2p2_b200 import _capi, synth

pytestmark = pytest.mark.gpu

POT = os.path.join(os.path.dirname(__file__), "golden", "potentials", "h2o_52")


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def _regular_entry(pos, elem, box):
    from n2p2_b200.mode import Prediction
    p = Prediction(POT)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_structure(pos, elem, box, remap=False)
    p.calculate_neighbor_list()
    out = p.neighbor_list()
    cutoff = p.get_max_cutoff_radius()
    p.close()
    return out, cutoff


def _oracle(pos, elem, box):
    """The reference's neighbor list and the positions it was built from:
    Structure::readFromLines remaps periodic structures (Structure.cpp:268,
    1223-1247), which recomputes every position from its fractional
    coordinates, so the other two lists are built from those positions."""
    from oracle.ref import RefModel
    ref = RefModel(POT)
    ref.setup_statistics()
    ref.set_structure(pos, elem, box)
    ref.evaluate(False)
    return ref.neighbors(), ref.positions()


def _noalloc(torch, pos, box, cutoff, capacity, expect=0):
    L = _capi.load()
    n = len(pos)
    dpos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    offsets = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    cap = max(capacity, 1)
    index = torch.zeros(cap, dtype=torch.int32, device="cuda")
    dr = torch.zeros((cap, 3), dtype=torch.float64, device="cuda")
    d = torch.zeros(cap, dtype=torch.float64, device="cuda")
    bp = None
    if box is not None:
        b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
        bp = b.ctypes.data_as(C.c_void_p)
    total = C.c_int64()
    err = C.create_string_buffer(256)
    rc = L.n2p2b_neighbor_list_noalloc(
        torch.cuda.current_device(), None, n, bp,
        C.c_void_p(dpos.data_ptr()), cutoff, C.c_void_p(counts.data_ptr()),
        C.c_void_p(offsets.data_ptr()), C.c_void_p(index.data_ptr()),
        C.c_void_p(dr.data_ptr()), C.c_void_p(d.data_ptr()), capacity,
        C.byref(total), err, 256)
    assert rc == expect, err.value.decode()
    if rc != 0:
        return total.value, err.value.decode()
    E = total.value
    return (counts.cpu().numpy().astype(np.int64),
            index[:E].cpu().numpy().astype(np.int64),
            dr[:E].cpu().numpy(), d[:E].cpu().numpy(),
            offsets.cpu().numpy())


def _same(a, b):
    c0, i0, r0, d0 = a[:4]
    c1, i1, r1, d1 = b[:4]
    assert np.array_equal(c0, c1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(r0.view(np.int64), r1.view(np.int64))
    assert np.array_equal(d0.view(np.int64), d1.view(np.int64))


def _skewed(nmol, seed):
    box, pos, elem = synth.water_box(nmol, seed)
    L = box[0, 0]
    cell = np.array([[L, 0.0, 0.0], [0.27 * L, 0.96 * L, 0.0],
                     [-0.18 * L, 0.21 * L, 1.03 * L]])
    frac = np.mod(pos / L, 1.0)
    return cell, frac @ cell, elem


def _inside(pos, box):
    return np.mod(pos @ np.linalg.inv(box), 1.0) @ box


def _cases():
    out = []
    box, pos, elem = synth.water_box(512, 21)      # 46.9 bohr: 3 cells
    out.append(("cells3", box, _inside(pos, box), elem, True))
    b2, p2, e2 = synth.water_box(134, 22)           # 30.0 bohr: 2 cells
    out.append(("cells2", b2, _inside(p2, b2), e2, True))
    b1, p1, e1 = synth.water_box(29, 23)            # 18.0 bohr: 1 cell
    out.append(("cells1", b1, _inside(p1, b1), e1, True))
    b0, p0, e0 = synth.water_box(4, 24)             # 9.4 bohr < cutoff
    out.append(("small_box", b0, _inside(p0, b0), e0, True))
    bs, ps, es = _skewed(128, 25)
    out.append(("skewed", bs, ps, es, True))
    bo, po, eo = synth.water_box(40, 26)
    out.append(("open", None, po, eo, True))
    bx, px, ex = synth.water_box(64, 27)
    px = _inside(px, bx)
    px[5] += bx[0]                                  # one atom outside
    out.append(("outside", bx, px, ex, False))
    return out


def test_noalloc_matches_regular_entry_point_and_oracle(torch):
    for name, box, pos, elem, oracle_ok in _cases():
        if oracle_ok:
            ref_list, pos = _oracle(pos, elem, box)
        reg, cutoff = _regular_entry(pos, elem, box)
        got = _noalloc(torch, pos, box, cutoff, int(reg[0].sum()) + 64)
        _same(reg, got)
        assert got[4][-1] == reg[0].sum(), name
        if oracle_ok:
            _same(ref_list, got)


def test_noalloc_two_calls_in_a_row(torch):
    box, pos, elem = synth.water_box(512, 21)
    frames = [_inside(pos, box),
              _inside(pos + np.random.default_rng(5).normal(0, 0.1,
                                                            pos.shape), box)]
    for fr in frames:
        reg, cutoff = _regular_entry(fr, elem, box)
        got = _noalloc(torch, fr, box, cutoff, int(reg[0].sum()) + 64)
        _same(reg, got)


def test_noalloc_capacity_one_short(torch):
    box, pos, elem = synth.water_box(64, 28)
    pos = _inside(pos, box)
    reg, cutoff = _regular_entry(pos, elem, box)
    need = int(reg[0].sum())
    total, msg = _noalloc(torch, pos, box, cutoff, need - 1,
                          expect=_capi.ERR_CAPACITY)
    assert total == need
    assert "capacity" in msg
    # the scratch is usable again right after the failed call
    got = _noalloc(torch, pos, box, cutoff, need)
    _same(reg, got)


def test_noalloc_rejects_oversized_input(torch):
    L = _capi.load()
    total = C.c_int64()
    err = C.create_string_buffer(256)
    box = np.eye(3).reshape(9) * 100.0
    rc = L.n2p2b_neighbor_list_noalloc(
        torch.cuda.current_device(), None, 1 << 20,
        box.ctypes.data_as(C.c_void_p), C.c_void_p(1), 12.0, C.c_void_p(1),
        C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), 0,
        C.byref(total), err, 256)
    assert rc == _capi.ERR_CAPACITY
    assert b"65536" in err.value
