"""GPU test of kw_spectral_derivative (the reference's staggered derivativeOperator,
Sources/KWave/Solver/KSpaceFirstOrder.swift:764-769, applied on its own) against numpy FP64, and
the spectral derivative of a sine (Tests/KWaveTests/FFTTests.swift:16-30)."""
import ctypes as C
import math

import numpy as np
import pytest

from kwave import abi
from kwave.runtime import Context

pytestmark = pytest.mark.gpu


def numpy_derivative(f, spacing, axis, shift):
    n = f.shape[axis]
    d = spacing[axis]
    val = 1.0 / (n * d)
    cutoff = (n - 1) // 2 + 1
    k = 2 * math.pi * np.concatenate([np.arange(cutoff), np.arange(-(n // 2), -(n // 2) + n - cutoff)]) * val
    op = 1j * k * np.exp(shift * 1j * k * d / 2)
    shp = [1] * f.ndim
    shp[axis] = n
    F = np.fft.fftn(f)
    return np.real(np.fft.ifftn(F * op.reshape(shp)))


def run_derivative(ctx, f, spacing, axis, shift, fn="kw_spectral_derivative"):
    import torch
    dim = f.ndim
    dims = list(f.shape) + [1] * (3 - dim)
    sp = list(spacing) + [1.0] * (3 - dim)
    t_in = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float32)).cuda()
    t_out = torch.empty_like(t_in)
    torch.cuda.synchronize()
    st = getattr(ctx.lib, fn)(ctx.h, dim, dims[0], dims[1], dims[2], sp[0], sp[1], sp[2], axis, shift,
                              C.c_void_p(t_in.data_ptr()), C.c_void_p(t_out.data_ptr()))
    if st != abi.KW_OK:
        raise RuntimeError(ctx.lib.kw_last_error_message(ctx.h).decode())
    torch.cuda.synchronize()
    return t_out.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("shape,axis,shift", [((64,), 0, 1), ((48, 40), 1, -1), ((40, 48), 0, 1),
                                              ((24, 20, 32), 2, 1), ((24, 20, 32), 0, -1), ((34, 27), 1, 1)])
def test_spectral_derivative_matches_numpy(shape, axis, shift):
    rng = np.random.default_rng(11)
    f = rng.standard_normal(shape).astype(np.float32)
    spacing = [1e-4 * (1 + 0.1 * a) for a in range(len(shape))]
    ctx = Context.default()
    out = run_derivative(ctx, f, spacing, axis, shift)
    ref = numpy_derivative(f.astype(np.float64), spacing, axis, shift)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err


def test_spectral_derivative_of_sine():
    # FFTTests.swift:16-30: d/dx sin(2 pi x / L) = (2 pi / L) cos(2 pi x / L) to 1e-3
    n, L = 64, 1.0
    dx = L / n
    x = np.arange(n) * dx
    f = np.sin(2 * math.pi * x / L)
    ctx = Context.default()
    # the staggered operator evaluates the derivative half a cell to the right
    out = run_derivative(ctx, f, [dx], 0, 1)
    expected = (2 * math.pi / L) * np.cos(2 * math.pi * (x + dx / 2) / L)
    assert np.max(np.abs(out - expected)) < 1e-3
