"""Python mirror of n2p2's Mode / Prediction interface over the C-ABI.

Method names follow nnp::Mode (libnnp/Mode.h:86-662) and nnp::Prediction
(libnnp/Prediction.h:27-40) in Python spelling; errors raised by the library
come back as the exception types the reference throws (std::runtime_error ->
RuntimeError, std::range_error / std::out_of_range -> IndexError,
std::invalid_argument -> ValueError).

Array arguments may be numpy arrays (host) or CUDA torch tensors (device);
device tensors are passed by pointer and never copied through the host.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi


class N2P2Error(RuntimeError):
    """A failed library call (message from n2p2b_last_error)."""

    def __init__(self, code: int, message: str):
        super().__init__(message.strip() or f"n2p2_b200 error {code}")
        self.code = code


class CapacityError(N2P2Error, IndexError):
    pass


class StateError(N2P2Error):
    pass


class ExtrapolationError(N2P2Error, IndexError):
    """An extrapolation warning with stop-on-warning set (the reference
    throws std::out_of_range); the evaluation's results are complete."""


def _is_device_tensor(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _ptr_and_loc(a, dtype):
    """(pointer, location, keepalive) for a host array or a CUDA tensor."""
    if _is_device_tensor(a):
        import torch
        want = torch.float64 if dtype == np.float64 else torch.int32
        if a.dtype != want or not a.is_contiguous():
            raise ValueError(f"device tensor must be contiguous {want}")
        return C.c_void_p(a.data_ptr()), _capi.DEVICE, a
    h = np.ascontiguousarray(a, dtype=dtype)
    return h.ctypes.data_as(C.c_void_p), _capi.HOST, h


class Mode:
    """nnp::Mode on one CUDA device."""

    def __init__(self, device: int = 0):
        self._L = _capi.load()
        h = C.c_void_p()
        rc = self._L.n2p2b_create(int(device), C.byref(h))
        if rc != 0:
            raise N2P2Error(rc, f"cannot create a context on CUDA device "
                                f"{device} (is a GPU visible?)")
        self._h = h
        self.num_atoms = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.n2p2b_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc == 0:
            return
        msg = (self._L.n2p2b_last_error(self._h) or b"").decode()
        if rc == _capi.ERR_CAPACITY:
            raise CapacityError(rc, msg)
        if rc == _capi.ERR_STATE:
            raise StateError(rc, msg)
        if rc == _capi.ERR_EXTRAPOLATION:
            raise ExtrapolationError(rc, msg)
        if rc == _capi.ERR_ARGUMENT:
            raise ValueError(msg)
        raise N2P2Error(rc, msg)

    # ---- setup (Mode.h) -------------------------------------------------
    def load_settings_file(self, path: str = "input.nn"):
        self._check(self._L.n2p2b_load_settings_file(self._h, path.encode()))

    def setup_generic(self):
        self._check(self._L.n2p2b_setup_generic(self._h))

    def setup_symmetry_function_scaling(self, path: str | None = "scaling.data"):
        self._check(self._L.n2p2b_setup_symmetry_function_scaling(
            self._h, path.encode() if path else None))

    def setup_symmetry_function_scaling_none(self):
        self.setup_symmetry_function_scaling(None)

    def setup_neural_network_weights(self, fmt: str = "weights.%03zu.data"):
        self._check(self._L.n2p2b_setup_neural_network_weights(
            self._h, fmt.encode()))

    # ---- potential queries ------------------------------------------------
    @property
    def num_elements(self) -> int:
        return self._L.n2p2b_num_elements(self._h)

    @property
    def elements(self) -> list[str]:
        out = []
        buf = C.create_string_buffer(8)
        for e in range(self.num_elements):
            self._check(self._L.n2p2b_element_symbol(self._h, e, buf, 8))
            out.append(buf.value.decode())
        return out

    def num_symmetry_functions(self, e: int) -> int:
        return self._L.n2p2b_num_symmetry_functions(self._h, e)

    def num_slots(self, e: int, ne: int) -> int:
        return self._L.n2p2b_num_slots(self._h, e, ne)

    def get_max_cutoff_radius(self) -> float:
        return self._L.n2p2b_max_cutoff_radius(self._h)

    def unit_conversion(self):
        """(normalizes, mean_energy, conv_energy, conv_length) of input.nn
        (0, 1, 1 without normalization)."""
        mean, ce, cl = C.c_double(), C.c_double(), C.c_double()
        flag = self._L.n2p2b_unit_conversion(self._h, C.byref(mean),
                                             C.byref(ce), C.byref(cl))
        return bool(flag == 1), mean.value, ce.value, cl.value

    def atomic_energy_offset(self, e: int) -> float:
        """Element::getAtomicEnergyOffset (atom_energy of input.nn)."""
        return self._L.n2p2b_atomic_energy_offset(self._h, e)

    def symmetry_function_params(self, e: int, s: int):
        """type, e1, e2, eta, rs, rc, zeta, lambda, scaling factor, line
        (Element::getSymmetryFunction(s), normalized units)."""
        out = (C.c_double * 10)()
        self._check(self._L.n2p2b_symmetry_function_params(self._h, e, s, out))
        return np.array(out[:])

    def symmetry_function_groups(self, e: int):
        """Member SF indices of every group of element e, in group order."""
        out = []
        for g in range(self._L.n2p2b_num_groups(self._h, e)):
            buf = (C.c_int32 * 256)()
            m = self._L.n2p2b_group_members(self._h, e, g, buf, 256)
            if m < 0:
                raise ValueError("bad group")
            out.append(list(buf[:m]))
        return out

    def element_indices(self, symbols) -> np.ndarray:
        m = {s: i for i, s in enumerate(self.elements)}
        return np.array([m[s] for s in symbols], dtype=np.int32)

    # ---- structure ---------------------------------------------------------
    def set_structure(self, positions, elements, box=None, remap: bool = True):
        """Atoms to evaluate (physical units); elements are element indices
        (or symbols), box is 3x3 lattice vectors as rows or None."""
        el = np.asarray(elements)
        if el.dtype.kind in "US":
            el = self.element_indices(el)
        el = np.ascontiguousarray(el, dtype=np.int32)
        n = len(el)
        p, loc, keep = _ptr_and_loc(positions, np.float64)
        bp = None
        if box is not None:
            b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
            bp = b.ctypes.data_as(C.c_void_p)
        self._check(self._L.n2p2b_set_structure(
            self._h, n, bp, p, loc,
            el.ctypes.data_as(C.POINTER(C.c_int32)),
            _capi.REMAP if remap else 0))
        self.num_atoms = n
        del keep

    def set_structures(self, structures, remap: bool = True):
        """A batch of independent structures, each (box or None, positions,
        elements); evaluated together, each exactly as alone."""
        counts = np.array([len(s[1]) for s in structures], dtype=np.int64)
        pos = np.ascontiguousarray(np.concatenate([s[1] for s in structures]),
                                   dtype=np.float64)
        el = np.ascontiguousarray(np.concatenate([s[2] for s in structures]),
                                  dtype=np.int32)
        periodic = [s[0] is not None for s in structures]
        if any(periodic) and not all(periodic):
            raise ValueError("a batch is all periodic or all open")
        bp = None
        if all(periodic):
            boxes = np.ascontiguousarray(
                np.stack([np.asarray(s[0], dtype=np.float64).reshape(9)
                          for s in structures]))
            bp = boxes.ctypes.data_as(C.c_void_p)
        self._check(self._L.n2p2b_set_structures(
            self._h, len(structures),
            counts.ctypes.data_as(C.POINTER(C.c_int64)), bp,
            pos.ctypes.data_as(C.c_void_p), _capi.HOST,
            el.ctypes.data_as(C.POINTER(C.c_int32)),
            _capi.REMAP if remap else 0))
        self.num_atoms = int(counts.sum())
        self.num_structures = len(structures)

    def structure_energies(self):
        out = np.zeros(getattr(self, "num_structures", 1))
        self._check(self._L.n2p2b_get_structure_energies(
            self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def capture_graph(self, use_forces: bool = True):
        self._check(self._L.n2p2b_capture_graph(self._h, int(use_forces)))

    def launch_graph(self):
        self._check(self._L.n2p2b_launch_graph(self._h))

    def autotune(self, use_forces: bool = True, repetitions: int = 3) -> str:
        buf = C.create_string_buffer(512)
        self._check(self._L.n2p2b_autotune(self._h, int(use_forces),
                                           int(repetitions), buf, 512))
        return buf.value.decode()

    def set_positions(self, positions):
        p, loc, keep = _ptr_and_loc(positions, np.float64)
        self._check(self._L.n2p2b_set_positions(self._h, p, loc))
        del keep

    # ---- evaluation (Mode.h) -----------------------------------------------
    def calculate_neighbor_list(self):
        self._check(self._L.n2p2b_calculate_neighbor_list(self._h))

    def calculate_symmetry_function_groups(self, derivatives: bool = True):
        self._check(self._L.n2p2b_calculate_symmetry_function_groups(
            self._h, int(derivatives)))

    def calculate_atomic_neural_networks(self, derivatives: bool = True):
        self._check(self._L.n2p2b_calculate_atomic_neural_networks(
            self._h, int(derivatives)))

    def calculate_energy(self):
        self._check(self._L.n2p2b_calculate_energy(self._h))

    def calculate_forces(self):
        self._check(self._L.n2p2b_calculate_forces(self._h))

    def evaluate_nnp(self, use_forces: bool = True):
        self._check(self._L.n2p2b_evaluate(self._h, int(use_forces)))

    def evaluate_async(self, use_forces: bool = True):
        self._check(self._L.n2p2b_evaluate_async(self._h, int(use_forces)))

    def finish(self):
        self._check(self._L.n2p2b_finish(self._h))

    def set_profiling(self, enable: bool = True):
        self._check(self._L.n2p2b_set_profiling(self._h, int(enable)))

    def stage_times(self, reset: bool = True):
        """Summed device ms per stage (NL, SF, NN, E, F) and run count."""
        ms = (C.c_double * 5)()
        runs = C.c_int64()
        self._check(self._L.n2p2b_get_stage_times(self._h, ms, C.byref(runs),
                                                  int(reset)))
        return list(ms), runs.value

    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.n2p2b_set_stream(
            self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    # ---- extrapolation warnings (Mode.h:209-224, 478-486) ----------------
    def setup_symmetry_function_statistics(self, collect_statistics=False,
                                           collect_extrapolation_warnings=False,
                                           write_extrapolation_warnings=False,
                                           stop_on_extrapolation_warnings=False):
        self._check(self._L.n2p2b_setup_symmetry_function_statistics(
            self._h, int(collect_statistics),
            int(collect_extrapolation_warnings),
            int(write_extrapolation_warnings),
            int(stop_on_extrapolation_warnings)))

    def get_num_extrapolation_warnings(self) -> int:
        return int(self._L.n2p2b_get_num_extrapolation_warnings(self._h))

    def reset_extrapolation_warnings(self):
        self._check(self._L.n2p2b_reset_extrapolation_warnings(self._h))

    def extrapolation_counts(self):
        """Warnings per atom of the last evaluation."""
        out = np.zeros(self.num_atoms, dtype=np.int32)
        self._check(self._L.n2p2b_get_extrapolation_counts(
            self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    # Record layout of n2p2b_extrapolation_warning (include/n2p2_b200.h).
    EW_DTYPE = np.dtype([("atom", np.int64), ("element", np.int32),
                         ("sf", np.int32), ("type", np.int32),
                         ("reserved", np.int32), ("value", np.float64),
                         ("gmin", np.float64), ("gmax", np.float64)])

    def extrapolation_warnings(self):
        """The warnings of the last evaluation as records (atom, element,
        sf (0-based), type, value, gmin, gmax), in the reference's order."""
        cnt = C.c_int64(0)
        self._check(self._L.n2p2b_get_extrapolation_warnings(
            self._h, 0, None, C.byref(cnt)))
        out = np.zeros(cnt.value, dtype=self.EW_DTYPE)
        if cnt.value:
            self._check(self._L.n2p2b_get_extrapolation_warnings(
                self._h, cnt.value, out.ctypes.data_as(C.c_void_p),
                C.byref(cnt)))
        return out

    # ---- distilled student ------------------------------------------------
    _STUDENT_MODES = {"off": _capi.STUDENT_OFF, "gated": _capi.STUDENT_GATED,
                      "only": _capi.STUDENT_ONLY}

    def setup_student(self, directory: str):
        """A student potential directory (same symmetry functions and
        scaling.data, its own weights and training_range.data)."""
        self._check(self._L.n2p2b_setup_student(self._h, directory.encode()))

    def set_student_mode(self, mode: str):
        """"off", "gated" (student; teacher for atoms outside the student's
        training range) or "only"."""
        self._check(self._L.n2p2b_set_student_mode(
            self._h, self._STUDENT_MODES[mode]))

    def student_gated_count(self) -> int:
        c = C.c_int64()
        self._check(self._L.n2p2b_get_student_gated_count(self._h,
                                                          C.byref(c)))
        return int(c.value)

    def student_train_step(self, energy_labels, force_labels, batch,
                           w_energy=1.0, w_force=1.0, lr=1e-3,
                           want_loss=False):
        """One Adam step; labels and batch are CUDA tensors (float64 atomic
        energies, float64 forces [n, 3], int32 atom indices)."""
        loss = (C.c_double * 2)() if want_loss else None
        self._check(self._L.n2p2b_student_train_step(
            self._h, C.c_void_p(energy_labels.data_ptr()),
            C.c_void_p(force_labels.data_ptr()), C.c_void_p(batch.data_ptr()),
            int(batch.numel()), float(w_energy), float(w_force), float(lr),
            loss))
        return (loss[0], loss[1]) if want_loss else None

    def student_reset_optimizer(self):
        self._check(self._L.n2p2b_student_reset_optimizer(self._h))

    def _student_blob(self, which, values=None):
        size = C.c_int64()
        self._check(self._L.n2p2b_student_weights(self._h, None, None,
                                                  C.byref(size), which))
        if values is None:
            out = np.zeros(size.value)
            self._check(self._L.n2p2b_student_weights(
                self._h, out.ctypes.data_as(C.POINTER(C.c_double)), None,
                None, which))
            return out
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self._L.n2p2b_student_weights(
            self._h, None, v.ctypes.data_as(C.POINTER(C.c_double)), None,
            which))

    def student_weights(self):
        return self._student_blob(0)

    def set_student_weights(self, blob):
        self._student_blob(0, blob)

    def student_gradient(self):
        return self._student_blob(1)

    def student_update_range(self, reset: bool = False):
        self._check(self._L.n2p2b_student_update_range(self._h, int(reset)))

    def student_write(self, directory: str):
        self._check(self._L.n2p2b_student_write(self._h, directory.encode()))

    _PRECISIONS = {"fp64": _capi.PRECISION_FP64,
                   "mixed": _capi.PRECISION_MIXED,
                   "bf16": _capi.PRECISION_BF16}

    def set_precision(self, mode: str):
        """"fp64" (plain form, default), "mixed" (FP32 symmetry functions;
        tensor-core NNs on BF16 high/low operand pairs with FP32
        accumulation) or "bf16" (the same with single BF16 operands).  The
        mixed forms keep FP64 displacements, energy sum and force
        accumulation."""
        if mode not in self._PRECISIONS:
            raise ValueError(f"unknown precision {mode!r}")
        self._check(self._L.n2p2b_set_precision(self._h,
                                                self._PRECISIONS[mode]))

    @property
    def precision(self) -> str:
        m = self._L.n2p2b_get_precision(self._h)
        return {v: k for k, v in self._PRECISIONS.items()}[m]

    # ---- results -----------------------------------------------------------
    @property
    def energy(self) -> float:
        e = C.c_double()
        self._check(self._L.n2p2b_get_energy(self._h, C.byref(e)))
        return e.value

    def forces(self, out=None):
        if out is not None and _is_device_tensor(out):
            self._check(self._L.n2p2b_get_forces(
                self._h, C.c_void_p(out.data_ptr()), _capi.DEVICE))
            return out
        f = np.zeros((self.num_atoms, 3))
        self._check(self._L.n2p2b_get_forces(
            self._h, f.ctypes.data_as(C.c_void_p), _capi.HOST))
        return f

    def atomic_energies(self):
        e = np.zeros(self.num_atoms)
        self._check(self._L.n2p2b_get_atomic_energies(
            self._h, e.ctypes.data_as(C.POINTER(C.c_double))))
        return e

    def neighbor_counts(self):
        c = np.zeros(self.num_atoms, dtype=np.int64)
        self._check(self._L.n2p2b_get_neighbor_counts(
            self._h, c.ctypes.data_as(C.POINTER(C.c_int64))))
        return c

    def neighbor_list(self):
        """(counts, index, dr, d) in the reference's list order."""
        cnt = self.neighbor_counts()
        E = int(cnt.sum())
        idx = np.zeros(E, dtype=np.int64)
        dr = np.zeros((E, 3))
        d = np.zeros(E)
        self._check(self._L.n2p2b_get_neighbor_list(
            self._h, idx.ctypes.data_as(C.POINTER(C.c_int64)),
            dr.ctypes.data_as(C.POINTER(C.c_double)),
            d.ctypes.data_as(C.POINTER(C.c_double))))
        return cnt, idx, dr, d

    def _max_sf(self):
        return max(self.num_symmetry_functions(e)
                   for e in range(self.num_elements))

    def _max_slots(self):
        ne = self.num_elements
        return max(self.num_slots(e, f) for e in range(ne) for f in range(ne))

    def symmetry_functions(self):
        s = self._max_sf()
        g = np.zeros((self.num_atoms, s))
        self._check(self._L.n2p2b_get_symmetry_functions(
            self._h, g.ctypes.data_as(C.POINTER(C.c_double)), s))
        return g

    def dEdG(self):
        s = self._max_sf()
        g = np.zeros((self.num_atoms, s))
        self._check(self._L.n2p2b_get_dEdG(
            self._h, g.ctypes.data_as(C.POINTER(C.c_double)), s))
        return g

    def dGdr(self):
        """(self [N, maxSF, 3], neighbor [E, maxSlots, 3])."""
        s = self._max_sf()
        sl = self._max_slots()
        E = int(self.neighbor_counts().sum())
        a = np.zeros((self.num_atoms, s, 3))
        b = np.zeros((E, sl, 3))
        self._check(self._L.n2p2b_get_dGdr(
            self._h, a.ctypes.data_as(C.POINTER(C.c_double)), s,
            b.ctypes.data_as(C.POINTER(C.c_double)), sl))
        return a, b


class Prediction(Mode):
    """nnp::Prediction: a potential directory with input.nn, scaling.data and
    weights.%03zu.data (libnnp/Prediction.cpp:26-76)."""

    def __init__(self, directory: str = ".", device: int = 0):
        super().__init__(device)
        self.directory = directory
        self.file_name_settings = os.path.join(directory, "input.nn")
        self.file_name_scaling = os.path.join(directory, "scaling.data")
        self.format_weights_files_short = os.path.join(directory,
                                                       "weights.%03zu.data")

    def setup(self):
        """Prediction::setup (libnnp/Prediction.cpp:34-46), including its
        setupSymmetryFunctionStatistics(false, false, true, false): write
        extrapolation warnings to stderr."""
        self.load_settings_file(self.file_name_settings)
        self.setup_generic()
        self.setup_symmetry_function_scaling(self.file_name_scaling)
        self.setup_neural_network_weights(self.format_weights_files_short)
        self.setup_symmetry_function_statistics(False, False, True, False)

    def predict(self, positions=None, elements=None, box=None):
        """Prediction::predict; with arguments, sets the structure first.
        Returns (energy, forces) in physical units."""
        if positions is not None:
            self.set_structure(positions, elements, box, remap=True)
        self.evaluate_nnp(True)
        return self.energy, self.forces()
