"""ctypes declarations of the C-ABI in include/n2p2_b200.h.

The library is the in-tree build n2p2_b200/libn2p2b200.so (``python -m
n2p2_b200.build``).  There is no fallback: importing this module without the
library raises, so a missing build can never silently turn into a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "libn2p2b200.so")

OK = 0
ERR_ARGUMENT = -1
ERR_SETUP = -2
ERR_CUDA = -3
ERR_CAPACITY = -4
ERR_STATE = -5
ERR_INTERNAL = -6
ERR_EXTRAPOLATION = -7
HOST = 0
DEVICE = 1
REMAP = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_BF16 = 2
STUDENT_OFF = 0
STUDENT_GATED = 1
STUDENT_ONLY = 2

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p

# name: (restype, argtypes)
SIGNATURES = {
    "n2p2b_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "n2p2b_destroy": (None, [_vp]),
    "n2p2b_last_error": (C.c_char_p, [_vp]),
    "n2p2b_set_stream": (C.c_int, [_vp, _vp]),
    "n2p2b_set_precision": (C.c_int, [_vp, C.c_int]),
    "n2p2b_get_precision": (C.c_int, [_vp]),
    "n2p2b_setup_symmetry_function_statistics": (
        C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "n2p2b_get_num_extrapolation_warnings": (C.c_int64, [_vp]),
    "n2p2b_reset_extrapolation_warnings": (C.c_int, [_vp]),
    "n2p2b_get_extrapolation_counts": (C.c_int, [_vp, _i32p]),
    "n2p2b_get_extrapolation_warnings": (C.c_int, [_vp, C.c_int64, _vp,
                                                   _i64p]),
    "n2p2b_set_structures": (C.c_int, [_vp, C.c_int64, _i64p, _vp, _vp,
                                       C.c_int, _i32p, C.c_int]),
    "n2p2b_get_structure_energies": (C.c_int, [_vp, _dp]),
    "n2p2b_capture_graph": (C.c_int, [_vp, C.c_int]),
    "n2p2b_launch_graph": (C.c_int, [_vp]),
    "n2p2b_autotune": (C.c_int, [_vp, C.c_int, C.c_int, C.c_char_p,
                                 C.c_size_t]),
    "n2p2b_setup_student": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_set_student_mode": (C.c_int, [_vp, C.c_int]),
    "n2p2b_get_student_gated_count": (C.c_int, [_vp, _i64p]),
    "n2p2b_student_train_step": (C.c_int, [
        _vp, _vp, _vp, _vp, C.c_int, C.c_double, C.c_double, C.c_double,
        _dp]),
    "n2p2b_student_reset_optimizer": (C.c_int, [_vp]),
    "n2p2b_student_weights": (C.c_int, [_vp, _dp, _dp, _i64p, C.c_int]),
    "n2p2b_student_update_range": (C.c_int, [_vp, C.c_int]),
    "n2p2b_student_write": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_load_settings_file": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_setup_generic": (C.c_int, [_vp]),
    "n2p2b_setup_symmetry_function_scaling": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_setup_neural_network_weights": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_setup": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_num_elements": (C.c_int, [_vp]),
    "n2p2b_element_symbol": (C.c_int, [_vp, C.c_int, C.c_char_p, C.c_size_t]),
    "n2p2b_element_index": (C.c_int, [_vp, C.c_char_p]),
    "n2p2b_num_symmetry_functions": (C.c_int, [_vp, C.c_int]),
    "n2p2b_num_slots": (C.c_int, [_vp, C.c_int, C.c_int]),
    "n2p2b_max_cutoff_radius": (C.c_double, [_vp]),
    "n2p2b_atomic_energy_offset": (C.c_double, [_vp, C.c_int]),
    "n2p2b_atomic_number": (C.c_int, [_vp, C.c_int]),
    "n2p2b_unit_conversion": (C.c_int, [_vp, _dp, _dp, _dp]),
    "n2p2b_set_neighbor_list": (C.c_int, [_vp, C.c_int64, _i32p, _i64p,
                                          _i64p, _i32p, _dp, C.c_int64]),
    "n2p2b_get_target_forces": (C.c_int, [_vp, _dp]),
    "n2p2b_symmetry_function_params": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "n2p2b_num_groups": (C.c_int, [_vp, C.c_int]),
    "n2p2b_group_members": (C.c_int, [_vp, C.c_int, C.c_int, _i32p, C.c_int]),
    "n2p2b_set_structure": (C.c_int, [_vp, C.c_int64, _vp, _vp, C.c_int,
                                      _i32p, C.c_int]),
    "n2p2b_set_positions": (C.c_int, [_vp, _vp, C.c_int]),
    "n2p2b_calculate_neighbor_list": (C.c_int, [_vp]),
    "n2p2b_calculate_symmetry_function_groups": (C.c_int, [_vp, C.c_int]),
    "n2p2b_calculate_atomic_neural_networks": (C.c_int, [_vp, C.c_int]),
    "n2p2b_calculate_energy": (C.c_int, [_vp]),
    "n2p2b_calculate_forces": (C.c_int, [_vp]),
    "n2p2b_evaluate": (C.c_int, [_vp, C.c_int]),
    "n2p2b_evaluate_async": (C.c_int, [_vp, C.c_int]),
    "n2p2b_finish": (C.c_int, [_vp]),
    "n2p2b_get_energy": (C.c_int, [_vp, _dp]),
    "n2p2b_get_forces": (C.c_int, [_vp, _vp, C.c_int]),
    "n2p2b_get_atomic_energies": (C.c_int, [_vp, _dp]),
    "n2p2b_get_neighbor_counts": (C.c_int, [_vp, _i64p]),
    "n2p2b_get_neighbor_list": (C.c_int, [_vp, _i64p, _dp, _dp]),
    "n2p2b_get_symmetry_functions": (C.c_int, [_vp, _dp, C.c_int]),
    "n2p2b_get_dEdG": (C.c_int, [_vp, _dp, C.c_int]),
    "n2p2b_get_dGdr": (C.c_int, [_vp, _dp, C.c_int, _dp, C.c_int]),
    "n2p2b_predict": (C.c_int, [_vp, C.c_int64, _vp, _vp, _i32p, _dp, _dp]),
    "n2p2b_set_profiling": (C.c_int, [_vp, C.c_int]),
    "n2p2b_get_stage_times": (C.c_int, [_vp, _dp, _i64p, C.c_int]),
    "n2p2b_kernel_launch_count": (C.c_uint64, []),
    "n2p2b_check_exp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "n2p2b_neighbor_list_noalloc": (C.c_int, [
        C.c_int, _vp, C.c_int64, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp,
        _vp, C.c_int64, _i64p, C.c_char_p, C.c_size_t]),
}

_lib = None


def load(path: str | None = None):
    """Loads the library and declares every exported symbol."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("N2P2B_LIBRARY") or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python -m n2p2_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib
