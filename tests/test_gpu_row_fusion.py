"""Row fusion: the register C2R of the velocity job also transforms the new u_a into the density
job's spectra, and the density C2R transforms rho0 div u and rho_sum into the power-law absorption
job's spectra (kw_jobs.cpp, kw_pass_rowr.cu), so those jobs skip their R2C.

Each absorption mode (power law with and without dispersion: two and one fused transforms; Stokes
and lossless: velocity fusion only) is run on grids whose row count leaves the last C2R tile
partly empty (rows past the end take part in the transforms' barriers only) and on a 128-point row
length (the benchmark's instantiation), against the FP64 oracle (relative L2 <= 1e-4 on the p
series and pFinal) and against the same run with fusion off (the default; the fused R2C uses
the C2R's radix split, so results agree to 1e-5 rather than bit for bit). A batch that mixes
an absorbing and a lossless simulation runs each one as it runs alone. Fusion is opt-in
(KW_FUSE_ROWS=1); the adjoint's fused reverse step is checked against the FP64 adjoint.
"""
import numpy as np
import pytest

import oracle
from cases import rel_l2
from kwave import (DescBuilder, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, RecordField,
                   SimulationOptions, SourceMode, toneBurst)
from kwave.api import AbsorptionMode
from kwave.runtime import Context
from test_gpu_parity import compare

pytestmark = pytest.mark.gpu

# (shape, pml): rows A*B against C2R rows per CTA (256 / (M / 8) for these half lengths M)
#   (100, 128): 100 rows, 32 per CTA;  (20, 22, 64): 440 rows, 64 per CTA;
#   (12, 14, 256): 168 rows, 16 per CTA (M = 128);  (13, 15, 256): 195 rows, so the last CTA's
#   second warp holds one row inside the grid and one past its end
SHAPES = [((100, 128), 6), ((20, 22, 64), 3), ((12, 14, 256), 2), ((13, 15, 256), 2)]
MODES = [AbsorptionMode.powerLaw, AbsorptionMode.noDispersion, AbsorptionMode.stokes, AbsorptionMode.noAbsorption]


def _case(shape, pml, mode, seed=7):
    rng = np.random.default_rng(seed)
    dim = len(shape)
    dx = 1e-4
    c = (1500 + 60 * rng.standard_normal(shape)).astype(np.float32)
    rho = (1000 + 40 * rng.standard_normal(shape)).astype(np.float32)
    args = []
    for n in shape:
        args += [n, dx]
    g = KWaveGrid(*args)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(40, g.dt)
    pm = np.zeros(shape, np.float32)
    pm[tuple([slice(pml + 1, n - pml - 1) for n in shape[:-1]] + [pml + 2])] = 1
    sig = (toneBurst(1 / g.dt, 2e6, 2) * 1e5).astype(np.float32)
    sm = np.zeros(shape, np.float32)
    sm[tuple([slice(None)] * (dim - 1) + [pml + 8])] = 1
    kw = dict(alphaCoeff=0.5, alphaPower=1.5, alphaMode=mode) if mode != AbsorptionMode.noAbsorption else {}
    med = KWaveMedium(c, rho, bOnA=5.0, **kw)
    return DescBuilder(g, med, KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                       KWaveSensor(mask=sm, record=RecordField.p | RecordField.pFinal), SimulationOptions(pmlSize=pml))


def _run(b):
    sim = Context.default().create_sim(b)
    try:
        sim.run()
        return {k: v for k, v in vars(sim.outputs()).items()}
    finally:
        sim.close()


@pytest.mark.parametrize("mode", MODES, ids=lambda m: m.name)
@pytest.mark.parametrize("shape,pml", SHAPES, ids=lambda v: str(v))
def test_fused_rows_match_oracle_and_unfused(shape, pml, mode, monkeypatch):
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    monkeypatch.setenv("KW_FUSE_ROWS", "1")
    b = _case(shape, pml, mode)
    fused = _run(b)
    ref, _ = oracle.run(b)
    compare(fused, ref)
    monkeypatch.setenv("KW_FUSE_ROWS", "0")
    plain = _run(b)
    for k in ("p", "pFinal"):
        assert rel_l2(fused[k], plain[k]) < 1e-5, (k, rel_l2(fused[k], plain[k]))


def test_batch_mixing_absorbing_and_lossless(monkeypatch):
    # the density C2R runs its fused variant for the whole launch; for the lossless member it
    # transforms nothing. The absorbing members run the same kernels as alone (bit for bit); the
    # lossless member's density update runs in the fused kernel instead of the plain one (the same
    # expressions, compiled in another kernel), so it is held to 1e-6
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    monkeypatch.setenv("KW_FUSE_ROWS", "1")
    builders = [_case((100, 128), 6, AbsorptionMode.powerLaw, seed=1), _case((100, 128), 6, AbsorptionMode.noAbsorption, seed=2),
                _case((100, 128), 6, AbsorptionMode.noDispersion, seed=3)]
    singles = [_run(b) for b in builders]
    batch = Context.default().create_batch(builders)
    try:
        batch.run()
        for i, b in enumerate(builders):
            npts = singles[i]["p"].shape[0]
            p, pf = batch.output(i, "p", b.grid.nt, npts), batch.output(i, "pFinal", b.grid.nt, npts)
            if i == 1:
                assert rel_l2(p, singles[i]["p"]) < 1e-6 and rel_l2(pf, singles[i]["pFinal"]) < 1e-6, i
            else:
                assert np.array_equal(p, singles[i]["p"]) and np.array_equal(pf, singles[i]["pFinal"]), i
    finally:
        batch.close()


@pytest.mark.parametrize("shape,kw", [((36, 32), dict(absorb="nodispersion", nonlinear=True, cartesian=False, nt=40, no_p0=True)),
                                      ((16, 20, 32), dict(absorb="powerlaw", nonlinear=True, cartesian=True, nt=30))])
def test_fused_adjoint_matches_fp64_adjoint(shape, kw, monkeypatch):
    # the forward fusions and the adjoint velocity C2R writing the summing job's spectra; 2D 36 x 32
    # puts rows inside and past the end of the grid into one warp of the last C2R tile
    from adjoint_cases import builder, problem
    monkeypatch.setenv("KW_FUSE_ROWS", "1")
    c, p0, data, kw = problem(shape, **kw)
    L, gc, gp = oracle.adjoint(builder(shape, c, p0, **kw), data)
    r = Context.default().adjoint(builder(shape, c, p0, **kw), data, grad_c0=True, grad_p0=p0 is not None)
    assert abs(r["misfit"] - L) <= 1e-3 * L, (r["misfit"], L)
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)
