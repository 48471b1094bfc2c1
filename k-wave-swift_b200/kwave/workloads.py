"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (no dataset is involved; numpy.random.default_rng(20261203 + config index)).

  ivp2d_128      128^2 homogeneous IVP, disc r5 p0 (smoothed), circle r40 sensor, nt 201
  hetero3d_256   256^3 heterogeneous nonlinear absorbing forward: 12 random spheres, alpha 0.75
                 dB/(MHz^1.5 cm), B/A 6, additive 1 MPa 1 MHz 3-cycle tone burst on a 64x64
                 plane at z = 30, sensor = full xy plane at z = 200 recording p and pMax
  batch2d_64     64 uneven 2D grids (n in {128,192,256,384,512}), smooth random c0 maps,
                 16-point line source, 256-point Cartesian circle sensor
  adjoint2d_512  512^2 adjoint gradient: 6 elliptical inclusions, power law y 1.1, smoothed p0
                 of 10 discs, 512-point Cartesian ring, 1500 steps, c0 perturbed by 1%
  adjoint3d_384  384^3 forward + adjoint: 3 layers + 8 spheres, power law y 1.5, B/A 5, 32x32
                 focused array at z = 25, 128x128 receive plane, 2000 steps, c0 perturbed by 1%
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


def _ellipses(shape, rng, count, c, s=1.0):
    nx, ny = shape
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    for _ in range(count):
        a, b = rng.uniform(10 * s, 60 * s, size=2)
        th = rng.uniform(0, math.pi)
        m = 20 + 30 * s
        cx, cy = rng.uniform(m, nx - m), rng.uniform(m, ny - m)
        xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
        yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
        c[(xr / a) ** 2 + (yr / b) ** 2 <= 1.0] = np.float32(rng.uniform(1420, 1600))


def adjoint2d(n: int = 512, steps: int = 1500):
    """The 2D adjoint-gradient configuration: returns (builder at the perturbed sound speed,
    builder at the true sound speed). 512^2, dx 0.1 mm, PML 20, `steps` time steps at
    dt = 0.3 dx / max(c_true); 6 elliptical inclusions (1420-1600 m/s) on 1500 m/s; rho 1000;
    power law alpha 0.5 dB/(MHz^1.1 cm), y = 1.1; p0 = a smoothed sum of 10 discs; a 512-point
    Cartesian ring of radius 240 dx recording p. The perturbed speed is c_true (1 + 0.01 N(0,1));
    c_ref is held at max(c_true) for both."""
    rng = np.random.default_rng(SEED + 3)
    dx = 1e-4
    shape = (n, n)
    s = n / 512.0
    c = np.full(shape, 1500.0, np.float32)
    _ellipses(shape, rng, 6, c, s)
    p0 = np.zeros(shape, np.float32)
    for _ in range(10):
        r = int(rng.integers(3, 13))
        cx, cy = (int(v) for v in rng.integers(n // 4, 3 * n // 4, size=2))
        p0 += makeDisc(n, n, cx, cy, r) * np.float32(rng.uniform(0.5, 1.5))
    p0 = _gauss_smooth_wrap(p0, 1.5).astype(np.float32)   # smooth stand-in: Gaussian sigma 1.5 points
    c_pert = (c * (1.0 + 0.01 * rng.standard_normal(shape))).astype(np.float32)
    c_ref = float(c.max())
    g = KWaveGrid(n, dx, n, dx)
    g.setTime(steps, 0.3 * dx / c_ref)
    sen = makeCartCircle(240 * s * dx, max(16, int(512 * s)))
    def mk(cc):
        med = KWaveMedium(cc, 1000.0, alphaCoeff=0.5, alphaPower=1.1, alphaMode=AbsorptionMode.powerLaw)
        return DescBuilder(g, med, KWaveSource(p0=p0), KWaveSensor(mask=sen, record=RecordField.p),
                           SimulationOptions(pmlSize=20, smoothP0=False, cRef=c_ref))
    return mk(c_pert), mk(c)


def adjoint3d(n: int = 384, steps: int = 2000):
    """The 3D forward + adjoint configuration: returns (builder at the perturbed sound speed,
    builder at the true one). 384^3, dx 0.15 mm, PML 20, `steps` time steps; three planar z-layers
    (c0 1480 / 1560 / 1620 m/s, rho0 1000 / 1050 / 1100, boundaries at z = n/3, 2n/3) with 8 random
    spheres as in the 256^3 forward; power law alpha 0.75 dB/(MHz^1.5 cm) with dispersion, B/A 5;
    a 32 x 32 array of single-point elements at pitch 4 on the plane z = 25, each a 1.5 MHz
    3-cycle burst delayed to focus at the grid centre (one signal row per element); a centred
    128 x 128 receive plane at z = 25 recording p. The perturbed speed is c_true (1 + 0.01 N(0,1));
    c_ref is held at max(c_true)."""
    rng = np.random.default_rng(SEED + 4)
    s = n / 384.0
    dx = 1.5e-4
    shape = (n, n, n)
    c = np.empty(shape, np.float32)
    rho = np.empty(shape, np.float32)
    z1, z2 = n // 3, 2 * n // 3
    for (lo, hi), cv, rv in (((0, z1), 1480.0, 1000.0), ((z1, z2), 1560.0, 1050.0), ((z2, n), 1620.0, 1100.0)):
        c[:, :, lo:hi] = cv
        rho[:, :, lo:hi] = rv
    _spheres(shape, rng, 8, max(2, int(round(8 * s))), max(3, int(round(30 * s))), int(round(20 * s)),
             int(round(20 * s)), c, rho, (1400.0, 1650.0), (900.0, 1100.0))
    c_ref = float(c.max())
    g = KWaveGrid(n, dx, n, dx, n, dx)
    g.makeTime(c_ref, cfl=0.3)
    g.setTime(steps, g.dt)
    # 32 x 32 elements at pitch 4 (scaled), centred, on z = 25 (scaled)
    ne = max(2, int(round(32 * s)))
    pitch = max(1, int(round(4 * s)))
    z_src = max(1, int(round(25 * s)))
    off = n // 2 - (ne * pitch) // 2
    pm = np.zeros(shape, np.float32)
    pos = []
    for i in range(ne):
        for j in range(ne):
            pm[off + i * pitch, off + j * pitch, z_src] = 1
            pos.append((off + i * pitch, off + j * pitch, z_src))
    # rows follow the ascending flat index of the mask: x major, then y (z fixed)
    pos.sort(key=lambda q: (q[0] * n + q[1]) * n + q[2])
    centre = np.array([n // 2, n // 2, n // 2], np.float64)
    dist = np.array([np.linalg.norm((np.array(q) - centre) * dx) for q in pos])
    delays = (dist.max() - dist) / 1500.0
    burst = toneBurst(1.0 / g.dt, 1.5e6, 3).astype(np.float64)
    shift = np.round(delays / g.dt).astype(int)
    length = len(burst) + int(shift.max())
    sig = np.zeros((len(pos), length), np.float32)
    for r, k in enumerate(shift):
        sig[r, k:k + len(burst)] = burst * 1e5
    sm = np.zeros(shape, np.float32)
    h = max(1, int(round(64 * s)))
    sm[n // 2 - h:n // 2 + h, n // 2 - h:n // 2 + h, z_src] = 1
    c_pert = (c * (1.0 + 0.01 * rng.standard_normal(shape))).astype(np.float32)

    def mk(cc):
        med = KWaveMedium(cc, rho, alphaCoeff=0.75, alphaPower=1.5, alphaMode=AbsorptionMode.powerLaw, bOnA=5.0)
        return DescBuilder(g, med, KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                           KWaveSensor(mask=sm, record=RecordField.p),
                           SimulationOptions(pmlSize=max(4, int(round(20 * s))), cRef=c_ref))
    return mk(c_pert), mk(c)
