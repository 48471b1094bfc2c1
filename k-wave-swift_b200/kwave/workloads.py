"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (no dataset is involved; numpy.random.default_rng(20261203 + config index)).

  ivp2d_128      128^2 homogeneous IVP, disc r5 p0 (smoothed), circle r40 sensor, nt 201
  hetero3d_256   256^3 heterogeneous nonlinear absorbing forward: 12 random spheres, alpha 0.75
                 dB/(MHz^1.5 cm), B/A 6, additive 1 MPa 1 MHz 3-cycle tone burst on a 64x64
                 plane at z = 30, sensor = full xy plane at z = 200 recording p and pMax
  batch2d_64     64 uneven 2D grids (n in {128,192,256,384,512}), smooth random c0 maps,
                 16-point line source, 256-point Cartesian circle sensor
"""
from __future__ import annotations

import math

import numpy as np

from .api import (AbsorptionMode, DescBuilder, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource,
                  RecordField, SimulationOptions, SourceMode)
from .shapes import makeCartCircle, makeCircle, makeDisc, toneBurst

SEED = 20261203


def ivp2d_128() -> DescBuilder:
    n = 128
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=4e-6)
    src = KWaveSource(p0=makeDisc(n, n, radius=5) * 1.0)
    sen = KWaveSensor(mask=makeCircle(n, n, radius=40), record=RecordField.p | RecordField.pFinal | RecordField.pMax)
    return DescBuilder(g, KWaveMedium(1500.0, 1000.0), src, sen, SimulationOptions(pmlSize=20, smoothP0=True))


def _spheres(shape, rng, count, r_lo, r_hi, lo_margin, hi_margin, c, rho, c_range, rho_range):
    n = shape[0]
    for _ in range(count):
        r = int(rng.integers(r_lo, r_hi + 1))
        cx, cy, cz = (int(v) for v in rng.integers(lo_margin + r, n - hi_margin - r + 1, size=3))
        cv = np.float32(rng.uniform(*c_range))
        rv = np.float32(rng.uniform(*rho_range))
        sl = tuple(slice(max(v - r, 0), min(v + r + 1, n)) for v in (cx, cy, cz))
        xs = np.arange(sl[0].start, sl[0].stop).reshape(-1, 1, 1) - cx
        ys = np.arange(sl[1].start, sl[1].stop).reshape(1, -1, 1) - cy
        zs = np.arange(sl[2].start, sl[2].stop).reshape(1, 1, -1) - cz
        m = (xs * xs + ys * ys + zs * zs) <= r * r
        c[sl][m] = cv
        rho[sl][m] = rv


def hetero3d(n: int = 256, steps: int | None = None) -> DescBuilder:
    """The 3D heterogeneous nonlinear absorbing forward (defaults to the 256^3 configuration)."""
    rng = np.random.default_rng(SEED + 1)
    dx = 1e-4
    shape = (n, n, n)
    c = np.full(shape, 1500.0, np.float32)
    rho = np.full(shape, 1000.0, np.float32)
    s = n / 256.0
    _spheres(shape, rng, 12, max(2, int(round(8 * s))), max(3, int(round(30 * s))), int(round(20 * s)),
             int(round(20 * s)), c, rho, (1400.0, 1650.0), (900.0, 1100.0))
    g = KWaveGrid(n, dx, n, dx, n, dx)
    g.makeTime(float(c.max()), cfl=0.3)
    # t_end = 1.2 x the time for a wave at the background speed to cross the domain
    t_end = 1.2 * (n * dx) / 1500.0
    nt = int(math.floor(t_end / g.dt)) + 1
    g.setTime(steps if steps is not None else nt, g.dt)
    pm = np.zeros(shape, np.float32)
    h = max(1, int(round(32 * s)))
    z_src = int(round(30 * s))
    pm[n // 2 - h:n // 2 + h, n // 2 - h:n // 2 + h, z_src] = 1
    sig = (toneBurst(1.0 / g.dt, 1e6, 3) * 1e6).astype(np.float32)
    sm = np.zeros(shape, np.float32)
    sm[:, :, int(round(200 * s))] = 1
    med = KWaveMedium(c, rho, alphaCoeff=0.75, alphaPower=1.5, alphaMode=AbsorptionMode.powerLaw, bOnA=6.0)
    return DescBuilder(g, med, KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                       KWaveSensor(mask=sm, record=RecordField.p | RecordField.pMax), SimulationOptions(pmlSize=20))


def _gauss_smooth_wrap(x: np.ndarray, sigma: float) -> np.ndarray:
    # Gaussian filter with wrap-around boundaries, done spectrally (separable Gaussian kernel).
    out = np.fft.fftn(x)
    for a, n in enumerate(x.shape):
        k = np.fft.fftfreq(n)
        g = np.exp(-2.0 * (math.pi * sigma * k) ** 2)
        shp = [1] * x.ndim
        shp[a] = n
        out = out * g.reshape(shp)
    return np.real(np.fft.ifftn(out))


def batch2d(count: int = 64, sizes=(128, 192, 256, 384, 512), steps: int | None = None) -> list[DescBuilder]:
    """Uneven 2D forwards: smooth random c0 maps, 16-point line source, 256-point Cartesian ring."""
    rng = np.random.default_rng(SEED + 2)
    dx = 1e-4
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        noise = rng.standard_normal((n, n))
        gsm = _gauss_smooth_wrap(noise, 4.0)
        c = (1500.0 + 50.0 * gsm / np.max(np.abs(gsm))).astype(np.float32)
        g = KWaveGrid(n, dx, n, dx)
        g.makeTime(float(c.max()), soundSpeedMin=float(c.min()), cfl=0.3)
        if steps is not None:
            g.setTime(min(steps, g.nt), g.dt)
        y0 = int(rng.integers(20, n - 36 + 1))
        pm = np.zeros((n, n), np.float32)
        pm[30, y0:y0 + 16] = 1
        sig = toneBurst(1.0 / g.dt, 2e6, 4).astype(np.float32)
        sen = makeCartCircle(0.35 * n * dx, 256)
        out.append(DescBuilder(g, KWaveMedium(c, 1000.0), KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                               KWaveSensor(mask=sen, record=RecordField.p), SimulationOptions(pmlSize=20)))
    return out
