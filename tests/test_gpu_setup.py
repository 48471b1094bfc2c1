"""Set-up paths of kw_sim_create: device blocks reused from destroyed simulations of the same
context (zeroed like fresh ones), host maps above 2 MiB staged through the context's pinned
buffers, and the reference sound speed taken as the device-side maximum of the c0 map.

A 96^3 heterogeneous power-law case (3.5 MB maps, so the staged path runs) against the FP64
oracle (relative L2 <= 1e-4 on p and pFinal), run three times on one context with other
simulations created and destroyed in between: the repeated runs equal the first bit for bit.
"""
import numpy as np
import pytest

import oracle
from kwave.runtime import Context
from test_gpu_parity import _reg_case, compare

pytestmark = pytest.mark.gpu


def _run(ctx, b):
    sim = ctx.create_sim(b)
    try:
        sim.run()
        return {k: v for k, v in vars(sim.outputs()).items()}
    finally:
        sim.close()


def test_reused_blocks_and_staged_maps(monkeypatch):
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    ctx = Context.default()
    b = _reg_case((96, 96, 96), 17, 8)
    first = _run(ctx, b)
    ref, _ = oracle.run(b)
    compare(first, ref)
    other = _reg_case((48, 40, 64), 5, 6)   # different sizes in between: blocks change hands
    for _ in range(2):
        _run(ctx, other)
        again = _run(ctx, b)
        for k, v in first.items():
            if v is not None:
                assert np.array_equal(again[k], v), k
