"""GPU test of n2p2b_neighbor_list_noalloc, the neighbor list for callers
that cannot allocate device memory while they run (for example an MD engine
that reserves all GPU memory at start-up and hands the library fixed
buffers).

The entry point is called through the C-ABI with buffers the test owns, twice
in a row on different frames (its static scratch is reused between the
calls), and each result must equal -- bit for bit, the tolerance of every
neighbor-list test here -- the list that the regular entry point
(n2p2b_calculate_neighbor_list) builds for the same positions.

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


def _reference_entry(pos, elem, box):
    from n2p2_b200.mode import Prediction
    p = Prediction(POT)
    p.setup()
    p.set_structure(pos, elem, box, remap=False)
    p.calculate_neighbor_list()
    out = p.neighbor_list()
    cutoff = p.get_max_cutoff_radius()
    p.close()
    return out, cutoff


def _noalloc(torch, pos, box, cutoff, capacity):
    L = _capi.load()
    n = len(pos)
    dpos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    offsets = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    index = torch.zeros(capacity, dtype=torch.int32, device="cuda")
    dr = torch.zeros((capacity, 3), dtype=torch.float64, device="cuda")
    d = torch.zeros(capacity, dtype=torch.float64, device="cuda")
    b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
    total = C.c_int64()
    err = C.create_string_buffer(256)
    rc = L.n2p2b_neighbor_list_noalloc(
        torch.cuda.current_device(), None, n, b.ctypes.data_as(C.c_void_p),
        C.c_void_p(dpos.data_ptr()), cutoff, C.c_void_p(counts.data_ptr()),
        C.c_void_p(offsets.data_ptr()), C.c_void_p(index.data_ptr()),
        C.c_void_p(dr.data_ptr()), C.c_void_p(d.data_ptr()), capacity,
        C.byref(total), err, 256)
    assert rc == 0, err.value.decode()
    E = total.value
    return (counts.cpu().numpy().astype(np.int64),
            index[:E].cpu().numpy().astype(np.int64),
            dr[:E].cpu().numpy(), d[:E].cpu().numpy(),
            offsets.cpu().numpy())


def test_noalloc_matches_regular_entry_point_twice(torch):
    box, pos, elem = synth.water_box(512, 21)
    L = box[0, 0]
    frames = [np.mod(pos, L),
              np.mod(pos + np.random.default_rng(5).normal(0, 0.1, pos.shape),
                     L)]
    for fr in frames:
        (c0, i0, r0, d0), cutoff = _reference_entry(fr, elem, box)
        c1, i1, r1, d1, off = _noalloc(torch, fr, box, cutoff,
                                       int(c0.sum()) + 64)
        assert np.array_equal(c0, c1)
        assert off[-1] == c0.sum()
        assert np.array_equal(i0, i1)
        assert np.array_equal(r0.view(np.int64), r1.view(np.int64))
        assert np.array_equal(d0.view(np.int64), d1.view(np.int64))


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
