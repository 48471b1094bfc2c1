"""GPU parity at the benchmark workloads' own grid sizes and time horizons.

The FP64 oracle's outputs for these runs are committed fixtures (tests/golden/long_*.npz, written by
tests/golden/make_long.py; tests/long_cases.py defines the cases and the kept subsample): the
3D heterogeneous nonlinear absorbing forward at 128^3 over its whole horizon (561 steps), the
256^3 configuration itself over its first 60 steps (the kernel instantiations the benchmark
times), and one member of each grid size of the uneven 2D batch over its whole horizon (643 to
2570 steps), run as one batch and, for the 512^2 member, also on its own.

Tolerances: relative L2 <= 1e-4 on the p series and on pFinal, <= 1e-3 on pMax (an aggregate).
At the end of a whole horizon most of the wave has left the grid and pFinal is a residual of
1e-5 .. 4e-4 of the peak pressure; there the FP32 rounding of the run (about 3e-8 of the peak)
is itself 1e-3 of the residual, so a residual final field (peak below 1 % of the peak sensor
pressure) is checked by its RMS error against the peak sensor pressure (<= 1e-6), and pFinal is
checked at 1e-4 relative L2 half way through the horizon (`*_mid` cases), where the wave is
inside the grid.
"""
import os

import numpy as np
import pytest

from cases import GOLDEN, rel_l2
from long_cases import CASES, batch_members, subsample
from kwave.runtime import Context

pytestmark = pytest.mark.gpu


def _fixture(name):
    z = np.load(os.path.join(GOLDEN, f"long_{name}.npz"))
    return {k: z[k] for k in z.files}


def _check(name, out, nt, p_peak=None):
    ref = _fixture(name)
    assert int(ref["nt"]) == nt
    got = subsample(CASES[name], out)
    errs = {}
    for k in ("p", "pMax", "pFinal"):
        if k not in ref:
            continue
        assert got[k].shape == ref[k].shape, (k, got[k].shape, ref[k].shape)
        assert np.abs(ref[k]).max() > 0, k
        errs[k] = rel_l2(got[k], ref[k])
    if "p" in errs:
        assert errs["p"] < 1e-4, f"{name} p: rel L2 {errs['p']:.3e}"
        if "pMax" in errs:
            assert errs["pMax"] < 1e-3, f"{name} pMax: rel L2 {errs['pMax']:.3e}"
        p_peak = float(np.abs(ref["p"]).max())
    pf = ref["pFinal"].astype(np.float64)
    if p_peak is not None and np.abs(pf).max() < 1e-2 * p_peak:
        rms = float(np.sqrt(np.mean((got["pFinal"] - pf) ** 2)))
        errs["pFinal_rms/p_peak"] = rms / p_peak
        assert rms / p_peak < 1e-6, f"{name} residual pFinal: RMS error {rms / p_peak:.3e} of the peak"
    else:
        assert errs["pFinal"] < 1e-4, f"{name} pFinal: rel L2 {errs['pFinal']:.3e}"
    print(f"\n{name}: nt {nt} " + " ".join(f"{k} {v:.2e}" for k, v in errs.items()))


def _run(builder):
    sim = Context.default().create_sim(builder)
    try:
        sim.run()
        return {k: v for k, v in vars(sim.outputs()).items()}
    finally:
        sim.close()


@pytest.mark.parametrize("name", ["hetero3d_128_full", "hetero3d_128_mid", "hetero3d_256_t60"])
def test_hetero3d_long(name):
    b = CASES[name]["build"]()
    _check(name, _run(b), b.grid.nt)


def test_batch_members_full_horizon():
    builders = batch_members()
    batch = Context.default().create_batch(builders)
    try:
        batch.run()
        for i, b in enumerate(builders):
            nt, npts = b.grid.nt, 256
            out = {"p": batch.output(i, "p", nt, npts), "pFinal": batch.output(i, "pFinal", nt, npts)}
            _check(f"batch2d_n{b.grid.shape[0]}_full", out, nt)
    finally:
        batch.close()


@pytest.mark.parametrize("n", [128, 192, 256, 384, 512])
def test_batch_member_mid_horizon(n):
    b = CASES[f"batch2d_n{n}_mid"]["build"]()
    _check(f"batch2d_n{n}_mid", _run(b), b.grid.nt)


def test_batch_member_512_alone():
    b = batch_members()[-1]
    assert b.grid.shape == (512, 512)
    _check("batch2d_n512_full", _run(b), b.grid.nt)
