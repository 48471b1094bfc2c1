"""ctypes mirror of include/kwave_cuda.h (the C ABI of the CUDA library).

Only plain C types cross this boundary: host pointers, sizes and enums. The structures here must
stay byte-for-byte identical to the header; ``tests/test_abi.py`` checks the layout.
"""
from __future__ import annotations

import ctypes as C

KW_ABI_VERSION = 2

# kw_status
KW_OK = 0
KW_ERR_INVALID = 1
KW_ERR_OOM = 2
KW_ERR_CUDA = 3
KW_ERR_NONFINITE = 4
KW_ERR_TIMEOUT = 5
KW_ERR_UNSUPPORTED = 6
KW_ERR_STATE = 7

STATUS_NAMES = {
    KW_OK: "KW_OK", KW_ERR_INVALID: "KW_ERR_INVALID", KW_ERR_OOM: "KW_ERR_OOM",
    KW_ERR_CUDA: "KW_ERR_CUDA", KW_ERR_NONFINITE: "KW_ERR_NONFINITE",
    KW_ERR_TIMEOUT: "KW_ERR_TIMEOUT", KW_ERR_UNSUPPORTED: "KW_ERR_UNSUPPORTED",
    KW_ERR_STATE: "KW_ERR_STATE",
}

# kw_sensor_kind
KW_SENSOR_NONE = 0
KW_SENSOR_BINARY = 1
KW_SENSOR_CARTESIAN = 2

# kw_field (SimulationOutput members, KSpaceFirstOrder.swift:47-73)
FIELDS = [
    "p", "pMax", "pMin", "pRms", "pFinal",
    "ux", "uy", "uz",
    "uxMax", "uyMax", "uzMax",
    "uxRms", "uyRms", "uzRms",
    "uxFinal", "uyFinal", "uzFinal",
    "ixAvg", "iyAvg", "izAvg",
]
FIELD_INDEX = {name: i for i, name in enumerate(FIELDS)}


class kw_array(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("len", C.c_size_t)]


class kw_signal(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("rows", C.c_int), ("len", C.c_int)]


class kw_sim_desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("dim", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dt", C.c_double),
        ("nt", C.c_int),
        ("pml_size", C.c_int),
        ("pml_alpha", C.c_double),
        ("smooth_p0", C.c_int), ("smooth_c0", C.c_int), ("smooth_rho0", C.c_int),
        ("c_ref", C.c_double),
        ("sound_speed", kw_array),
        ("density", kw_array),
        ("alpha_coeff", kw_array),
        ("alpha_power", C.c_double),
        ("alpha_mode", C.c_int),
        ("b_on_a", kw_array),
        ("p0", C.POINTER(C.c_float)),
        ("p_mask", C.POINTER(C.c_float)),
        ("p", kw_signal),
        ("p_mode", C.c_int),
        ("u_mask", C.POINTER(C.c_float)),
        ("ux", kw_signal), ("uy", kw_signal), ("uz", kw_signal),
        ("u_mode", C.c_int),
        ("sensor_kind", C.c_int),
        ("sensor_mask", C.POINTER(C.c_float)),
        ("sensor_points", C.c_int),
        ("record", C.c_uint),
        ("directivity_angle", C.POINTER(C.c_float)),
        ("directivity_size", C.c_double),
        ("directivity_pattern", C.c_int),
        ("axisymmetric", C.c_int),
    ]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_int, C.c_int, C.c_void_p)
MONITOR_FN = C.CFUNCTYPE(None, C.c_int, C.POINTER(C.c_float), C.c_size_t, C.c_void_p)


class kw_callbacks(C.Structure):
    _fields_ = [
        ("progress", PROGRESS_FN),
        ("monitor", MONITOR_FN),
        ("monitor_interval", C.c_int),
        ("user", C.c_void_p),
    ]


class kw_kernel_timing(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("ms", C.c_double), ("bytes", C.c_double)]


class kw_adjoint_desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int),
        ("data", C.POINTER(C.c_float)),
        ("policy", C.c_int),
        ("checkpoint_interval", C.c_int),
        ("memory_budget", C.c_double),
        ("grad_c0", C.POINTER(C.c_float)),
        ("grad_p0", C.POINTER(C.c_float)),
        ("grad_rho0", C.POINTER(C.c_float)),
        ("misfit", C.c_double),
        ("forward_ms", C.c_double),
        ("reverse_ms", C.c_double),
        ("interval", C.c_int),
        ("checkpoints", C.c_int),
    ]


KW_CHECKPOINT_SQRT, KW_CHECKPOINT_INTERVAL, KW_CHECKPOINT_BUDGET, KW_CHECKPOINT_STORE_ALL = 0, 1, 2, 3
KW_CHECKPOINT_REVOLVE = 4

# Every symbol include/kwave_cuda.h declares, with its ctypes signature.
P = C.c_void_p
SIGNATURES = {
    "kw_sim_desc_init": (None, [C.POINTER(kw_sim_desc)]),
    "kw_version": (C.c_char_p, []),
    "kw_abi_version": (C.c_int, []),
    "kw_context_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "kw_context_set_stream": (C.c_int, [P, P]),
    "kw_context_destroy": (None, [P]),
    "kw_last_error_message": (C.c_char_p, [P]),
    "kw_sim_create": (C.c_int, [P, C.POINTER(kw_sim_desc), C.POINTER(P)]),
    "kw_sim_run": (C.c_int, [P, C.POINTER(kw_callbacks)]),
    "kw_sim_reset": (C.c_int, [P]),
    "kw_sim_step": (C.c_int, [P, C.c_int]),
    "kw_sim_synchronize": (C.c_int, [P]),
    "kw_sim_current_step": (C.c_int, [P, C.POINTER(C.c_int)]),
    "kw_sim_num_sensor_points": (C.c_int, [P, C.POINTER(C.c_int)]),
    "kw_sim_output_size": (C.c_int, [P, C.c_int, C.POINTER(C.c_size_t)]),
    "kw_sim_get_output": (C.c_int, [P, C.c_int, C.POINTER(C.c_float), C.c_size_t]),
    "kw_sim_device_field": (C.c_int, [P, C.c_int, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_size_t)]),
    "kw_sim_destroy": (None, [P]),
    "kw_sim_profile_step": (C.c_int, [P, C.c_int, C.POINTER(kw_kernel_timing), C.c_int, C.POINTER(C.c_int)]),
    "kw_spectral_derivative": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_int, C.c_int, P, P]),
    "kw_spectral_derivative_noalloc": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                 C.c_double, C.c_int, C.c_int, P, P]),
    "kw_adjoint_desc_init": (None, [C.POINTER(kw_adjoint_desc)]),
    "kw_adjoint_run": (C.c_int, [P, C.POINTER(kw_sim_desc), C.POINTER(kw_adjoint_desc)]),
    "kw_batch_create": (C.c_int, [P, C.POINTER(kw_sim_desc), C.c_int, C.POINTER(P)]),
    "kw_batch_run": (C.c_int, [P, C.POINTER(kw_callbacks)]),
    "kw_batch_reset": (C.c_int, [P]),
    "kw_batch_step": (C.c_int, [P, C.c_int]),
    "kw_batch_synchronize": (C.c_int, [P]),
    "kw_batch_output_size": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
    "kw_batch_get_output": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_size_t]),
    "kw_batch_destroy": (None, [P]),
}


def bind(lib: C.CDLL, signatures: dict = SIGNATURES) -> C.CDLL:
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
