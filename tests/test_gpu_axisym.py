"""Axisymmetric solver (kspaceFirstOrderAS) on the GPU against the numpy golden cases and the FP64
oracle: relative L2 <= 1e-4 on the p time series and pFinal, as ParityAxisymmetricTests.swift
(which checks 1e-4 against the maximum), for the IVP, additive and Dirichlet pressure sources,
Stokes absorption, B/A, additive ux / uy sources and a heterogeneous medium; a larger grid whose
expanded rows take the register kernels; the reference's preconditions."""
import numpy as np
import pytest

import oracle
from cases import GOLDEN_AS_CASES, builder_from_case, load_golden, rel_l2
from kwave import (AbsorptionMode, DescBuilder, KWaveError, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource,
                   RecordField, SimulationOptions, abi, kspaceFirstOrderAS, makeDisc)
from kwave.runtime import Context

pytestmark = pytest.mark.gpu


def run_gpu(builder):
    sim = Context.default().create_sim(builder)
    try:
        sim.run()
        return sim.output("p"), sim.output("pFinal")
    finally:
        sim.close()


@pytest.mark.parametrize("name", GOLDEN_AS_CASES)
def test_axisymmetric_golden_case(name):
    case, ref = load_golden(name)
    p, pf = run_gpu(builder_from_case(case))
    assert p.shape == ref["p"].shape and pf.shape == ref["pFinal"].shape
    assert rel_l2(p, ref["p"]) < 1e-4, rel_l2(p, ref["p"])
    assert rel_l2(pf, ref["pFinal"]) < 1e-4, rel_l2(pf, ref["pFinal"])


def test_axisymmetric_larger_grid_and_api():
    # 128 x 64 (expanded rows of 256 points), smoothed p0 disc on the axis, heterogeneous speed
    nx, ny = 128, 64
    rng = np.random.default_rng(11)
    c = (1500 + 30 * rng.standard_normal((nx, ny))).astype(np.float32)
    g = KWaveGrid(nx, 1e-4, ny, 1e-4)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(120, g.dt)
    p0 = np.zeros((nx, ny), np.float32)
    p0[60:68, 0:5] = 1.0
    sm = np.zeros((nx, ny), np.float32)
    sm[100, 0:40:3] = 1
    med = KWaveMedium(c, 1000.0, alphaCoeff=0.5, alphaMode=AbsorptionMode.stokes, bOnA=6.0)
    opts = SimulationOptions(pmlSize=12)
    b = DescBuilder(g, med, KWaveSource(p0=p0), KWaveSensor(mask=sm, record=RecordField.p), opts, axisymmetric=True)
    ref, _ = oracle.run(b)
    p, pf = run_gpu(b)
    assert np.abs(ref["p"]).max() > 0
    assert rel_l2(p, ref["p"]) < 1e-4 and rel_l2(pf, ref["pFinal"]) < 1e-4
    out = kspaceFirstOrderAS(g, med, KWaveSource(p0=p0), KWaveSensor(mask=sm, record=RecordField.p), opts)
    assert np.array_equal(out.p, p) and np.array_equal(out.pFinal, pf)


def test_axisymmetric_preconditions():
    g = KWaveGrid(32, 1e-4, 16, 1e-4)
    g.setTime(10, 2e-8)
    sen = KWaveSensor(mask=np.ones((32, 16), np.float32))
    with pytest.raises(KWaveError) as e:   # power-law absorption is not axisymmetric in k-Wave
        kspaceFirstOrderAS(g, KWaveMedium(1500.0, 1000.0, alphaCoeff=0.5, alphaPower=1.5,
                                          alphaMode=AbsorptionMode.powerLaw),
                           KWaveSource(p0=makeDisc(32, 16, radius=2)), sen)
    assert e.value.status == abi.KW_ERR_INVALID
    with pytest.raises(KWaveError) as e:   # no source
        kspaceFirstOrderAS(g, KWaveMedium(1500.0, 1000.0), KWaveSource(), sen)
    assert e.value.status == abi.KW_ERR_INVALID
