"""ctypes binding of the C ABI declared in include/kwave_b200.h.

The structures below mirror the C declarations field by field.  The library is
loaded from this package directory (``libkwave_b200.so``, built in-tree); when
it is missing the import raises -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_NAME = "libkwave_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

KW_ABI_VERSION = 3

KW_OK = 0
KW_ERR_INVALID = 1
KW_ERR_CUDA = 2
KW_ERR_NOMEM = 3
KW_ERR_UNSUPPORTED = 4
KW_ERR_TIMEOUT = 5

REC_BITS = {
    "p": 0, "p_max": 1, "p_min": 2, "p_rms": 3, "p_max_all": 4, "p_min_all": 5, "p_final": 6,
    "u": 7, "u_max": 8, "u_min": 9, "u_rms": 10, "u_max_all": 11, "u_min_all": 12, "u_final": 13,
    "u_non_staggered": 14,
}

SOURCE_MODES = {"dirichlet": 0, "additive-no-correction": 1, "additive": 2}
KW_LOSSLESS, KW_ABSORBING, KW_STOKES = 0, 1, 2
KW_COLUMN_MAJOR, KW_ROW_MAJOR = 0, 1
ALPHA_MODES = {None: 0, "no_absorption": 1, "no_dispersion": 2}

KCLASS = {"zstage_u": 0, "zstage_r": 1, "zstage_p": 2, "ypass": 3, "xpass": 4, "sensor": 5, "source": 6}

f32p = C.POINTER(C.c_float)
u64p = C.POINTER(C.c_uint64)


class KWaveError(RuntimeError):
    """Raised for every non-zero kw_status; ``status`` holds the code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class kw_source(C.Structure):
    _fields_ = [
        ("num_time_samples", C.c_uint64),
        ("mode", C.c_int32),
        ("num_points", C.c_uint64),
        ("index", u64p),
        ("num_signals", C.c_uint64),
        ("signal_index", u64p),
        ("input", f32p),
    ]


class kw_transducer_source(C.Structure):
    _fields_ = [("num_points", C.c_uint64), ("index", u64p), ("delay", u64p), ("apodization", f32p),
                ("signal_length", C.c_uint64), ("input_signal", f32p)]


class kw_problem(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("dim", C.c_int32),
        ("Nx", C.c_uint64), ("Ny", C.c_uint64), ("Nz", C.c_uint64),
        ("Nt", C.c_uint64),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("c_ref", C.c_double),
        ("c0", f32p), ("c0_scalar", C.c_double),
        ("rho0", f32p), ("rho0_scalar", C.c_double),
        ("rho0_sgx", f32p), ("rho0_sgy", f32p), ("rho0_sgz", f32p),
        ("pml_x_size", C.c_uint64), ("pml_y_size", C.c_uint64), ("pml_z_size", C.c_uint64),
        ("pml_x_alpha", C.c_double), ("pml_y_alpha", C.c_double), ("pml_z_alpha", C.c_double),
        ("use_kspace", C.c_int32),
        ("use_sg", C.c_int32),
        ("nonlinear_flag", C.c_int32),
        ("BonA", f32p), ("BonA_scalar", C.c_double),
        ("absorbing_flag", C.c_int32),
        ("alpha_coeff", f32p), ("alpha_coeff_scalar", C.c_double),
        ("alpha_power", C.c_double),
        ("alpha_mode", C.c_int32),
        ("alpha_sign", C.c_double * 2),
        ("p_source", kw_source),
        ("u_source", kw_source * 3),
        ("p0_source_input", f32p),
        ("sensor_num", C.c_uint64),
        ("sensor_mask_index", u64p),
        ("record_start_index", C.c_uint64),
        ("record", C.c_uint32),
        ("time_reversal_input", f32p),
        ("inside_lo", C.c_uint64 * 3),
        ("inside_hi", C.c_uint64 * 3),
        ("device", C.c_int32),
        ("array_order", C.c_int32),
        ("derive_rho0_sg", C.c_int32),
        ("sensor_vertices", C.c_uint32),
        ("sensor_weights", f32p),
        ("alpha_filter", f32p),
        ("transducer_source", kw_transducer_source),
        ("stream_to_disk", C.c_uint64),
        ("stream_to_disk_file", C.c_char_p),
    ]


class kw_output_desc(C.Structure):
    _fields_ = [
        ("sensor_num", C.c_uint64),
        ("num_time_points", C.c_uint64),
        ("inside_shape", C.c_uint64 * 3),
        ("grid_shape", C.c_uint64 * 3),
    ]


class kw_outputs(C.Structure):
    _fields_ = [
        ("p", f32p), ("p_max", f32p), ("p_min", f32p), ("p_rms", f32p),
        ("p_max_all", f32p), ("p_min_all", f32p), ("p_final", f32p),
        ("u", f32p * 3), ("u_max", f32p * 3), ("u_min", f32p * 3), ("u_rms", f32p * 3),
        ("u_max_all", f32p * 3), ("u_min_all", f32p * 3),
        ("u_final", f32p * 3), ("u_non_staggered", f32p * 3),
    ]


# every symbol the header declares, with its signature
class kw_server_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("max_active", C.c_int32),
                ("steps_per_slice", C.c_int32), ("request_timeout_ms", C.c_uint32), ("fill_cells", C.c_uint64)]


class kw_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("failed", C.c_uint64), ("active", C.c_uint64), ("pending", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("cell_steps", C.c_double), ("busy_seconds", C.c_double),
                ("setup_seconds", C.c_double), ("issue_seconds", C.c_double), ("retire_seconds", C.c_double),
                ("wait_seconds", C.c_double)]


SYMBOLS = {
    "kw_last_error": (C.c_char_p, []),
    "kw_abi_version": (C.c_int, []),
    "kw_plan_create": (C.c_int, [C.POINTER(kw_problem), C.POINTER(C.c_void_p)]),
    "kw_plan_outputs": (C.c_int, [C.c_void_p, C.POINTER(kw_output_desc)]),
    "kw_run": (C.c_int, [C.c_void_p, C.POINTER(kw_outputs)]),
    "kw_reset": (C.c_int, [C.c_void_p]),
    "kw_run_device": (C.c_int, [C.c_void_p]),
    "kw_copy_outputs": (C.c_int, [C.c_void_p, C.POINTER(kw_outputs)]),
    "kw_step": (C.c_int, [C.c_void_p, C.c_uint64]),
    "kw_plan_destroy": (C.c_int, [C.c_void_p]),
    "kw_set_timing": (C.c_int, [C.c_void_p, C.c_uint32]),
    "kw_get_timing": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "kw_plan_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "kw_run_timed": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "kw_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "kw_gradient_noalloc": (C.c_int, [C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int32,
                                      C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "kw_plan_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "kw_set_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "kw_adjoint_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "kw_keep_checkpoints": (C.c_int, [C.c_void_p, C.c_int32, C.c_uint32]),
    "kw_server_create": (C.c_int, [C.POINTER(kw_server_config), C.POINTER(C.c_void_p)]),
    "kw_server_submit": (C.c_int, [C.c_void_p, C.POINTER(kw_problem), C.POINTER(C.c_uint64)]),
    "kw_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(kw_outputs), C.POINTER(C.c_double)]),
    "kw_server_wait_for": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(kw_outputs),
                                     C.POINTER(C.c_double)]),
    "kw_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(kw_server_stats)]),
    "kw_server_destroy": (C.c_int, [C.c_void_p]),
}

_lib = None


def load_library(path=None):
    """Load the in-tree shared library (raises OSError when it is absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError("%s not found: build it with `python __graft_entry__.py build` "
                      "(no CPU fallback exists)" % p)
    lib = C.CDLL(p)
    for name, (res, args) in SYMBOLS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status):
    if status != KW_OK:
        msg = load_library().kw_last_error().decode(errors="replace")
        raise KWaveError(status, msg or ("kw_status %d" % status))


def fptr(a):
    """Pointer to a C-contiguous float32 array (None -> NULL)."""
    if a is None:
        return f32p()
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(f32p)


def uptr(a):
    if a is None:
        return u64p()
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(u64p)
