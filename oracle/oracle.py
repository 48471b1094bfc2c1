"""ctypes loader for the FP64 oracle (oracle/_build/libkwref.so). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module. It runs
the same kw_sim_desc the CUDA library receives through a double-precision restatement of
k-wave-swift's kspaceFirstOrder (oracle/kwref.cpp) and returns float64 outputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libkwref.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        from kwave import abi
        L = C.CDLL(LIB)
        L.kwref_run.restype = C.c_int
        L.kwref_run.argtypes = [C.POINTER(abi.kw_sim_desc), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.kwref_run_timed.restype = C.c_int
        L.kwref_run_timed.argtypes = [C.POINTER(abi.kw_sim_desc), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.kwref_output_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
        L.kwref_get_output.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        L.kwref_free.argtypes = [C.c_void_p]
        L.kwref_free.restype = None
        L.kwref_last_error.restype = C.c_char_p
        L.kwref_loop_seconds.restype = C.c_double
        L.kwref_loop_seconds.argtypes = [C.c_void_p]
        L.kwref_steps_done.argtypes = [C.c_void_p]
        L.kwref_fft.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        L.kwref_pml_profile.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.kwref_smooth.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.kwref_smoothing_window.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.kwref_adjoint.restype = C.c_int
        L.kwref_adjoint.argtypes = [C.POINTER(abi.kw_sim_desc), C.POINTER(C.c_double), C.c_int,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
        L.kwref_db2neper.restype = C.c_double
        L.kwref_db2neper.argtypes = [C.c_double, C.c_double]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def run(builder, nthreads: int = 0, max_steps: int = -1, timed_from: int = 0):
    """Run the oracle on a kwave.DescBuilder; returns (dict of float64 outputs, loop seconds)
    (kspaceFirstOrderAS when the descriptor's axisymmetric flag is set). The loop seconds cover
    the time steps from `timed_from` on (the earlier ones are untimed warm-up steps)."""
    from kwave import abi
    from kwave.api import output_shape
    L = lib()
    h = C.c_void_p()
    st = L.kwref_run_timed(C.byref(builder.desc), int(nthreads), int(max_steps), int(timed_from), C.byref(h))
    if st != 0:
        raise OracleError(f"status {st}: {L.kwref_last_error().decode()}")
    try:
        steps = L.kwref_steps_done(h)
        out = {}
        n_sensor = None
        for name in abi.FIELDS:
            n = C.c_size_t()
            L.kwref_output_size(h, abi.FIELD_INDEX[name], C.byref(n))
            if n.value == 0:
                out[name] = None
                continue
            a = np.empty(n.value)
            L.kwref_get_output(h, abi.FIELD_INDEX[name], _dp(a), n.value)
            out[name] = a
        # sensor count from an aggregate or series
        for name in ("p", "ux"):
            if out.get(name) is not None and steps > 0:
                n_sensor = out[name].size // steps
        for name in abi.FIELDS:
            if out[name] is not None:
                ns = n_sensor if n_sensor is not None else out[name].size
                out[name] = out[name].reshape(output_shape(name, builder.shape, ns, steps, out[name].size))
        return out, L.kwref_loop_seconds(h)
    finally:
        L.kwref_free(h)


def adjoint(builder, data: np.ndarray, nthreads: int = 0, grad_rho0: bool = False):
    """FP64 discrete adjoint: (misfit, dL/dc0, dL/dp0) of L = 1/2 sum (p_sensor - data)^2, with
    `data` shaped like the p series [n_sensor, nt]; with grad_rho0, (misfit, dL/dc0, dL/dp0,
    dL/drho0)."""
    L = lib()
    d = np.ascontiguousarray(data, dtype=np.float64)
    shape = builder.shape
    gc = np.zeros(int(np.prod(shape)))
    gp = np.zeros(int(np.prod(shape)))
    gr = np.zeros(int(np.prod(shape))) if grad_rho0 else None
    mis = C.c_double()
    st = L.kwref_adjoint(C.byref(builder.desc), _dp(d), int(nthreads), C.byref(mis), _dp(gc), _dp(gp),
                         _dp(gr) if grad_rho0 else None)
    if st != 0:
        raise OracleError(f"status {st}: {L.kwref_last_error().decode()}")
    if grad_rho0:
        return mis.value, gc.reshape(shape), gp.reshape(shape), gr.reshape(shape)
    return mis.value, gc.reshape(shape), gp.reshape(shape)


def fft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    re = np.ascontiguousarray(x.real.copy())
    im = np.ascontiguousarray(x.imag.copy())
    lib().kwref_fft(len(x), _dp(re), _dp(im), int(inverse))
    return re + 1j * im


def pml_profile(n, dx, dt, c, m, alpha, staggered) -> np.ndarray:
    out = np.empty(n)
    st = lib().kwref_pml_profile(n, dx, dt, c, m, alpha, int(staggered), _dp(out))
    if st != 0:
        raise OracleError("invalid pml")
    return out


def smooth(field: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(np.asarray(field, dtype=np.float64))
    dims = (C.c_int * f.ndim)(*f.shape)
    out = np.empty_like(f)
    lib().kwref_smooth(f.ndim, dims, _dp(f), _dp(out))
    return out


def smoothing_window(shape) -> np.ndarray:
    dims = (C.c_int * len(shape))(*shape)
    out = np.empty(shape)
    lib().kwref_smoothing_window(len(shape), dims, _dp(out))
    return out


def db2neper(alpha: float, y: float) -> float:
    return lib().kwref_db2neper(alpha, y)
