"""Long-horizon and full-size parity cases: the benchmark workloads at their own grid sizes and time
horizons, with sensors chosen so that the FP64 oracle's outputs fit in small committed fixtures.

Each case names a builder and the subsample the fixture keeps:
  rows      sensor rows kept (slice over the sensor's row order)
  t_stride  every t_stride-th time sample of the kept rows
  final     the slices of pFinal kept (a sub-lattice of the full field)
The GPU test records every row and sample and compares the same subsample, so the relative L2
errors are those of the kept entries (an unbiased sample of the full outputs).

`tests/golden/make_long.py` writes the fixtures `tests/golden/long_<name>.npz` from the oracle.
"""
from __future__ import annotations

import copy

import numpy as np

from kwave import DescBuilder, KWaveSensor, RecordField, workloads


def _with_sensor(b: DescBuilder, mask, record) -> DescBuilder:
    return DescBuilder(b.grid, b.medium, b.source, KWaveSensor(mask=mask, record=record), b.options)


def _first_steps(b: DescBuilder, steps: int) -> DescBuilder:
    """The same simulation stopped after `steps` time steps."""
    g = copy.copy(b.grid)
    g.setTime(steps, b.grid.dt)
    return DescBuilder(g, b.medium, b.source, b.sensor, b.options)


def hetero3d_128_full() -> DescBuilder:
    """The 3D heterogeneous nonlinear absorbing forward at 128^3 over its whole time horizon
    (1.2 transit times, 561 steps): 16 x 16 sensor points on the receive plane z = 100."""
    b = workloads.hetero3d(128)
    m = np.zeros(b.shape, np.float32)
    m[::8, ::8, 100] = 1
    return _with_sensor(b, m, RecordField.p | RecordField.pMax)


def hetero3d_256_t60() -> DescBuilder:
    """The 256^3 benchmark configuration itself (the kernels the benchmark times), first 60 steps:
    the tone burst is still being injected; sensor points on two planes either side of the source
    plane z = 30."""
    b = workloads.hetero3d(256, steps=60)
    m = np.zeros(b.shape, np.float32)
    m[64:192:8, 64:192:8, 24] = 1
    m[64:192:8, 64:192:8, 36] = 1
    return _with_sensor(b, m, RecordField.p | RecordField.pMax)


def batch_members() -> list[DescBuilder]:
    """The first simulation of each grid size of the 64-simulation uneven batch, full time horizon
    (643 ... 2570 steps), with its 256-point Cartesian ring sensor."""
    seen = {}
    for b in workloads.batch2d():
        seen.setdefault(b.grid.shape[0], b)
    return [seen[n] for n in sorted(seen)]


# `*_full` cases keep the p series of the whole horizon and the final field, `*_mid` ones the
# field half way through (while the wave is still inside the grid: at the end of a full horizon
# the final field is a residual of 1e-5 .. 4e-4 of the peak pressure).
CASES = {
    "hetero3d_128_full": dict(build=hetero3d_128_full, rows=slice(None), t_stride=4,
                              final=(slice(None, None, 4),) * 3),
    "hetero3d_128_mid": dict(build=lambda: _first_steps(hetero3d_128_full(), 280), rows=slice(None), t_stride=4,
                             final=(slice(None, None, 4),) * 3, series=False),
    "hetero3d_256_t60": dict(build=hetero3d_256_t60, rows=slice(None), t_stride=1,
                             final=(slice(80, 176, 2), slice(80, 176, 2), slice(14, 46, 2))),
}
for _i, _n in enumerate((128, 192, 256, 384, 512)):
    CASES[f"batch2d_n{_n}_full"] = dict(build=(lambda i=_i: batch_members()[i]), rows=slice(None, None, 4),
                                        t_stride=4, final=(slice(None, None, 4),) * 2)
    CASES[f"batch2d_n{_n}_mid"] = dict(
        build=(lambda i=_i: (lambda b: _first_steps(b, b.grid.nt // 2))(batch_members()[i])),
        rows=slice(None, None, 4), t_stride=4, final=(slice(None, None, 4),) * 2, series=False)


def subsample(case: dict, out: dict) -> dict:
    """The kept entries of an output dict (p series, pMax, pFinal), as float32."""
    r = {}
    if case.get("series", True) and out.get("p") is not None:
        r["p"] = np.ascontiguousarray(out["p"][case["rows"], ::case["t_stride"]], dtype=np.float32)
    if case.get("series", True) and out.get("pMax") is not None:
        r["pMax"] = np.ascontiguousarray(out["pMax"][case["rows"]], dtype=np.float32)
    r["pFinal"] = np.ascontiguousarray(out["pFinal"][case["final"]], dtype=np.float32)
    return r
