"""The allocation-free spectral derivative must give the allocating entry point's result.

kw_spectral_derivative_noalloc exists for callers that cannot allocate device memory: a host whose
own memory manager already holds the GPU's memory, or a loop that cannot take cudaMalloc/cudaFree's
device-wide synchronisation. It takes all of its scratch from one fixed 16 MiB device array that
every call shares, so these tests call it several times in a row and compare each result with
kw_spectral_derivative, which allocates its scratch, on the same input. They also check that a
problem too large for the fixed array is refused with a clear message. This file is collected last
so that a failure here cannot hide the result of any other test.
"""
import ctypes as C

import numpy as np
import pytest

from kwave import abi
from kwave.runtime import Context

pytestmark = pytest.mark.gpu

TOL = 1e-5   # relative L2, the tolerance of the derivative tests


def _call(ctx, fn, t_in, t_out, shape, spacing, axis, shift):
    dims = list(shape) + [1] * (3 - len(shape))
    sp = list(spacing) + [1.0] * (3 - len(spacing))
    return getattr(ctx.lib, fn)(ctx.h, len(shape), dims[0], dims[1], dims[2], sp[0], sp[1], sp[2], axis, shift,
                                C.c_void_p(t_in.data_ptr()), C.c_void_p(t_out.data_ptr()))


def _both(ctx, f, spacing, axis, shift):
    import torch
    t_in = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float32)).cuda()
    ref = torch.full_like(t_in, float("nan"))
    out = torch.full_like(t_in, float("nan"))
    torch.cuda.synchronize()
    st = _call(ctx, "kw_spectral_derivative", t_in, ref, f.shape, spacing, axis, shift)
    assert st == abi.KW_OK, ctx.lib.kw_last_error_message(ctx.h).decode()
    st = _call(ctx, "kw_spectral_derivative_noalloc", t_in, out, f.shape, spacing, axis, shift)
    assert st == abi.KW_OK, ctx.lib.kw_last_error_message(ctx.h).decode()
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64), ref.cpu().numpy().astype(np.float64)


def test_noalloc_matches_allocating_entry_point_call_after_call():
    ctx = Context.default()
    rng = np.random.default_rng(5)
    cases = [((64, 48), [1e-4, 1.2e-4], 0, 1), ((24, 20, 32), [1e-4] * 3, 2, -1), ((64, 48), [1e-4, 1.2e-4], 1, -1)]
    for shape, spacing, axis, shift in cases:   # consecutive calls share (and reuse) the scratch
        f = rng.standard_normal(shape)
        out, ref = _both(ctx, f, spacing, axis, shift)
        assert np.all(np.isfinite(out))
        err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
        assert err < TOL, (shape, axis, err)


def test_noalloc_refuses_problems_beyond_its_scratch():
    import torch
    ctx = Context.default()
    shape = (4096, 1024)          # half-spectrum of 4096 x 514 complex values needs > 16 MiB
    t_in = torch.zeros(shape, device="cuda")
    t_out = torch.zeros(shape, device="cuda")
    torch.cuda.synchronize()
    st = _call(ctx, "kw_spectral_derivative_noalloc", t_in, t_out, shape, [1e-4, 1e-4], 0, 1)
    assert st == abi.KW_ERR_INVALID
    msg = ctx.lib.kw_last_error_message(ctx.h).decode()
    assert "allocation-free scratch" in msg and str(16 * 1024 * 1024) in msg
