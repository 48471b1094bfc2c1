"""Loader and thin object wrappers for libkwave_cuda.so (the CUDA library's C ABI).

The library is built in-tree by ``k-wave-swift_b200/build.py`` into ``k-wave-swift_b200/_build``.
There is no fallback: if the library is missing or no CUDA device is usable, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Callable, Optional, Sequence

import numpy as np

from . import abi
from .api import DescBuilder, KWaveError, SimulationOutput, output_shape

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("KWAVE_CUDA_LIB") or os.path.join(_PKG_DIR, "_build", "libkwave_cuda.so")

_lib: Optional[C.CDLL] = None
_lock = threading.Lock()


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load and bind libkwave_cuda.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise KWaveError(abi.KW_ERR_UNSUPPORTED,
                                 f"CUDA library not built: {path} (run k-wave-swift_b200/build.py)")
            _lib = abi.bind(C.CDLL(path))
        return _lib


def _check(lib: C.CDLL, ctx, status: int) -> None:
    if status != abi.KW_OK:
        msg = lib.kw_last_error_message(ctx)
        raise KWaveError(status, msg.decode() if msg else "")


class Context:
    _default: Optional["Context"] = None

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.kw_context_create(device, C.byref(h))
        if st != abi.KW_OK:
            raise KWaveError(st, self.lib.kw_last_error_message(None).decode() or "kw_context_create failed")
        self.h = h
        self._owned = True

    @classmethod
    def default(cls) -> "Context":
        if cls._default is None:
            cls._default = Context(0)
            cls._default._owned = False
        return cls._default

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self._owned:
            self.close()

    def close(self) -> None:
        if self.h:
            self.lib.kw_context_destroy(self.h)
            self.h = C.c_void_p()

    def set_stream(self, stream_handle: int) -> None:
        _check(self.lib, self.h, self.lib.kw_context_set_stream(self.h, C.c_void_p(stream_handle)))

    def create_sim(self, builder: DescBuilder) -> "Simulation":
        return Simulation(self, builder)

    def create_batch(self, builders: Sequence[DescBuilder]) -> "Batch":
        return Batch(self, builders)

    def adjoint(self, builder: DescBuilder, data: np.ndarray, grad_c0: bool = True, grad_p0: bool = False,
                policy: int = abi.KW_CHECKPOINT_SQRT, interval: int = 0, memory_budget: float = 0.0,
                grad_rho0: bool = False) -> dict:
        """kw_adjoint_run: misfit 1/2 sum (p_sensor - data)^2 and its gradients (see the header)."""
        d = np.ascontiguousarray(data, dtype=np.float32)
        shape = builder.shape
        a = abi.kw_adjoint_desc()
        self.lib.kw_adjoint_desc_init(C.byref(a))
        a.data = d.ctypes.data_as(C.POINTER(C.c_float))
        a.policy = int(policy)
        a.checkpoint_interval = int(interval)
        a.memory_budget = float(memory_budget)
        gc = np.zeros(shape, np.float32) if grad_c0 else None
        gp = np.zeros(shape, np.float32) if grad_p0 else None
        gr = np.zeros(shape, np.float32) if grad_rho0 else None
        if gr is not None:
            a.grad_rho0 = gr.ctypes.data_as(C.POINTER(C.c_float))
        if gc is not None:
            a.grad_c0 = gc.ctypes.data_as(C.POINTER(C.c_float))
        if gp is not None:
            a.grad_p0 = gp.ctypes.data_as(C.POINTER(C.c_float))
        _check(self.lib, self.h, self.lib.kw_adjoint_run(self.h, C.byref(builder.desc), C.byref(a)))
        return {"misfit": a.misfit, "grad_c0": gc, "grad_p0": gp, "grad_rho0": gr, "forward_ms": a.forward_ms,
                "reverse_ms": a.reverse_ms, "interval": a.interval, "checkpoints": a.checkpoints}


def _callbacks(progress, monitor, interval, shape):
    keep = []
    cb = abi.kw_callbacks()
    if progress is not None:
        f = abi.PROGRESS_FN(lambda t, nt, u: progress(t, nt))
        keep.append(f)
        cb.progress = f
    if monitor is not None:
        def _mon(t, ptr, count, u):
            arr = np.ctypeslib.as_array(ptr, shape=(count,)).copy().reshape(shape)
            monitor(t, arr)
        f2 = abi.MONITOR_FN(_mon)
        keep.append(f2)
        cb.monitor = f2
    cb.monitor_interval = int(interval)
    return cb, keep


class Simulation:
    def __init__(self, ctx: Context, builder: DescBuilder):
        self.ctx, self.lib, self.builder = ctx, ctx.lib, builder
        h = C.c_void_p()
        _check(self.lib, ctx.h, self.lib.kw_sim_create(ctx.h, C.byref(builder.desc), C.byref(h)))
        self.h = h

    def run(self, progress: Optional[Callable] = None, monitor: Optional[Callable] = None,
            monitor_interval: int = 1) -> None:
        cb, keep = _callbacks(progress, monitor, monitor_interval, self.builder.shape)
        _check(self.lib, self.ctx.h, self.lib.kw_sim_run(self.h, C.byref(cb)))
        del keep

    def reset(self) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_sim_reset(self.h))

    def step(self, n: int) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_sim_step(self.h, int(n)))

    def synchronize(self) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_sim_synchronize(self.h))

    @property
    def t(self) -> int:
        v = C.c_int()
        _check(self.lib, self.ctx.h, self.lib.kw_sim_current_step(self.h, C.byref(v)))
        return v.value

    @property
    def n_sensor(self) -> int:
        v = C.c_int()
        _check(self.lib, self.ctx.h, self.lib.kw_sim_num_sensor_points(self.h, C.byref(v)))
        return v.value

    def output(self, name: str) -> Optional[np.ndarray]:
        f = abi.FIELD_INDEX[name]
        n = C.c_size_t()
        _check(self.lib, self.ctx.h, self.lib.kw_sim_output_size(self.h, f, C.byref(n)))
        if n.value == 0:
            return None
        out = np.empty(n.value, dtype=np.float32)
        _check(self.lib, self.ctx.h,
               self.lib.kw_sim_get_output(self.h, f, out.ctypes.data_as(C.POINTER(C.c_float)), n.value))
        return out.reshape(output_shape(name, self.builder.shape, self.n_sensor, self.t, n.value))

    def outputs(self) -> SimulationOutput:
        o = SimulationOutput()
        for name in abi.FIELDS:
            setattr(o, name, self.output(name))
        return o

    def profile_step(self, reps: int = 3) -> list[dict]:
        """Per-launch mean device time (ms) and algorithmic bytes of one time step."""
        buf = (abi.kw_kernel_timing * 256)()
        n = C.c_int()
        _check(self.lib, self.ctx.h, self.lib.kw_sim_profile_step(self.h, int(reps), buf, 256, C.byref(n)))
        return [{"name": buf[i].name.decode(), "ms": buf[i].ms, "bytes": buf[i].bytes} for i in range(n.value)]

    def close(self) -> None:
        if self.h:
            self.lib.kw_sim_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent simulations stepped together (kw_batch_*)."""

    def __init__(self, ctx: Context, builders: Sequence[DescBuilder]):
        self.ctx, self.lib, self.builders = ctx, ctx.lib, list(builders)
        arr = (abi.kw_sim_desc * len(self.builders))(*[b.desc for b in self.builders])
        self._arr = arr
        h = C.c_void_p()
        _check(self.lib, ctx.h, self.lib.kw_batch_create(ctx.h, arr, len(self.builders), C.byref(h)))
        self.h = h

    def run(self, progress: Optional[Callable] = None) -> None:
        cb, keep = _callbacks(progress, None, 1, None)
        _check(self.lib, self.ctx.h, self.lib.kw_batch_run(self.h, C.byref(cb)))
        del keep

    def reset(self) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_batch_reset(self.h))

    def step(self, n: int) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_batch_step(self.h, int(n)))

    def synchronize(self) -> None:
        _check(self.lib, self.ctx.h, self.lib.kw_batch_synchronize(self.h))

    def output(self, i: int, name: str, steps: int, n_sensor: int) -> Optional[np.ndarray]:
        f = abi.FIELD_INDEX[name]
        n = C.c_size_t()
        _check(self.lib, self.ctx.h, self.lib.kw_batch_output_size(self.h, i, f, C.byref(n)))
        if n.value == 0:
            return None
        out = np.empty(n.value, dtype=np.float32)
        _check(self.lib, self.ctx.h, self.lib.kw_batch_get_output(
            self.h, i, f, out.ctypes.data_as(C.POINTER(C.c_float)), n.value))
        return out.reshape(output_shape(name, self.builders[i].shape, n_sensor, steps, n.value))

    def close(self) -> None:
        if self.h:
            self.lib.kw_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
