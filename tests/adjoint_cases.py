"""Small adjoint test problems shared by the oracle (CPU) and device (GPU) adjoint tests."""
import numpy as np

import oracle
from kwave import (AbsorptionMode, DescBuilder, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource,
                   RecordField, SimulationOptions, makeCartCircle, toneBurst)

DT = 1.5e-8


def density(shape, seed=1):
    """The heterogeneous density of `builder` (fixed seed)."""
    rng = np.random.default_rng(seed)
    return (1000 + 30 * rng.standard_normal(shape)).astype(np.float32)


def builder(shape, c, p0, absorb="none", nonlinear=False, source=True, cartesian=True, nt=50, seed=1, rho=None):
    """Heterogeneous medium (fixed seed, or the density `rho`), optional power-law / Stokes
    absorption and B/A, an initial pressure p0 (or None) and an additive line source, a Cartesian
    ring or binary sensor row."""
    dim = len(shape)
    args = []
    for n in shape:
        args += [n, 1e-4]
    g = KWaveGrid(*args)
    g.setTime(nt, DT)
    rho = density(shape, seed) if rho is None else np.asarray(rho, np.float32)
    kw = {}
    if absorb == "powerlaw":
        kw = dict(alphaCoeff=0.5, alphaPower=1.5, alphaMode=AbsorptionMode.powerLaw)
    elif absorb == "nodispersion":
        kw = dict(alphaCoeff=0.5, alphaPower=1.3, alphaMode=AbsorptionMode.noDispersion)
    elif absorb == "stokes":
        kw = dict(alphaCoeff=0.5, alphaMode=AbsorptionMode.stokes)
    if nonlinear:
        kw["bOnA"] = 5.0
    med = KWaveMedium(np.asarray(c, np.float32), rho, **kw)
    srckw = {}
    if p0 is not None:
        srckw["p0"] = np.asarray(p0, np.float32)
    if source:
        pm = np.zeros(shape, np.float32)
        idx = [shape[0] // 4] + [slice(shape[a] // 3, shape[a] // 3 + 5) for a in range(1, dim)]
        if dim == 1:
            idx = [shape[0] // 4]
        pm[tuple(idx)] = 1
        srckw.update(pMask=pm, p=(toneBurst(1 / DT, 3e6, 2) * 2e4).astype(np.float32))
    if cartesian and dim >= 2:
        r = 0.3 * min(shape) * 1e-4
        if dim == 2:
            sen = KWaveSensor(mask=makeCartCircle(r, 12), record=RecordField.p)
        else:
            pts = makeCartCircle(r, 12)
            sen = KWaveSensor(mask=np.vstack([pts, np.full((1, 12), 1e-4, np.float32)]).astype(np.float32),
                              record=RecordField.p)
    else:
        sm = np.zeros(shape, np.float32)
        idx = [int(0.7 * shape[0])] + [slice(2, shape[a] - 2, 3) for a in range(1, dim)]
        sm[tuple(idx)] = 1
        sen = KWaveSensor(mask=sm, record=RecordField.p)
    return DescBuilder(g, med, KWaveSource(**srckw), sen, SimulationOptions(pmlSize=4, cRef=1600.0, smoothP0=False))


def problem(shape, seed=5, **kw):
    """(c, p0, data) with data recorded by the FP64 oracle at a perturbed sound speed."""
    rng = np.random.default_rng(seed)
    c = (1500 + 40 * rng.standard_normal(shape)).astype(np.float32).astype(np.float64)
    p0 = np.zeros(shape)
    sl = tuple(slice(n // 2 - 2, n // 2 + 2) for n in shape)
    p0[sl] = 3e5
    if kw.get("no_p0"):
        p0 = None
    kw = {k: v for k, v in kw.items() if k != "no_p0"}
    ctrue = c + 30 * rng.standard_normal(shape)
    data = oracle.run(builder(shape, ctrue, p0, **kw))[0]["p"]
    return c, p0, data, kw


def fd_misfit_diff(shape, c, p0, data, v, eps, which, kw):
    """Central difference L(x + eps v) - L(x - eps v) of the FP64 oracle misfit, with the exact
    float32 perturbation that the descriptor arrays see."""
    base = c if which == "c" else (p0 if which == "p" else density(shape).astype(np.float64))
    xp = (base + eps * v).astype(np.float32).astype(np.float64)
    xm = (base - eps * v).astype(np.float32).astype(np.float64)
    if which == "c":
        lp = oracle.adjoint(builder(shape, xp, p0, **kw), data)[0]
        lm = oracle.adjoint(builder(shape, xm, p0, **kw), data)[0]
    elif which == "rho":
        lp = oracle.adjoint(builder(shape, c, p0, rho=xp, **kw), data)[0]
        lm = oracle.adjoint(builder(shape, c, p0, rho=xm, **kw), data)[0]
    else:
        lp = oracle.adjoint(builder(shape, c, xp, **kw), data)[0]
        lm = oracle.adjoint(builder(shape, c, xm, **kw), data)[0]
    return lp - lm, xp - xm
