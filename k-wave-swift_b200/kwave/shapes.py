"""Input builders used to set up simulations: binary masks, Cartesian point sets and tone bursts.

These are caller-side helpers of k-wave-swift, restated with numpy so that the same arrays feed
both the CUDA library and the oracle. Each follows the reference function it names:

  makeDisc        Sources/KWave/Geometry/Shapes.swift:14-23
  makeCircle      Sources/KWave/Geometry/Shapes.swift:32-61
  makeBall        Sources/KWave/Geometry/Shapes.swift:64-78
  makeCartCircle  Sources/KWave/Geometry/CartesianShapes.swift:53-68
  gaussian        Sources/KWave/Signal/Generation.swift:10-13
  toneBurst       Sources/KWave/Signal/Generation.swift:29-49
"""
from __future__ import annotations

import math

import numpy as np


def _default_center(n: int) -> int:
    # Shapes.swift:6 — 0-based grid centre n/2 (k-Wave's floor(N/2)+1, 1-based).
    return n // 2


def makeDisc(nx: int, ny: int, cx: int | None = None, cy: int | None = None, radius: float = 1.0) -> np.ndarray:
    """Filled disc mask [nx, ny] (float32 0/1); distances evaluated in float32 like the reference."""
    cx = _default_center(nx) if cx is None else cx
    cy = _default_center(ny) if cy is None else cy
    xs = np.arange(nx, dtype=np.float32).reshape(nx, 1)
    ys = np.arange(ny, dtype=np.float32).reshape(1, ny)
    dx2 = (xs - np.float32(cx)) * (xs - np.float32(cx))
    dy2 = (ys - np.float32(cy)) * (ys - np.float32(cy))
    r2 = dx2 + dy2
    return (r2 <= np.float32(radius * radius)).astype(np.float32)


def makeBall(nx: int, ny: int, nz: int, cx: int | None = None, cy: int | None = None,
             cz: int | None = None, radius: float = 1.0) -> np.ndarray:
    """Filled ball mask [nx, ny, nz] (float32 0/1)."""
    cx = _default_center(nx) if cx is None else cx
    cy = _default_center(ny) if cy is None else cy
    cz = _default_center(nz) if cz is None else cz
    xs = np.arange(nx, dtype=np.float32).reshape(nx, 1, 1)
    ys = np.arange(ny, dtype=np.float32).reshape(1, ny, 1)
    zs = np.arange(nz, dtype=np.float32).reshape(1, 1, nz)
    d2 = ((xs - np.float32(cx)) ** 2 + (ys - np.float32(cy)) ** 2) + (zs - np.float32(cz)) ** 2
    return (d2 <= np.float32(radius * radius)).astype(np.float32)


def makeCircle(nx: int, ny: int, cx: int | None = None, cy: int | None = None,
               radius: float = 1.0, arcAngle: float | None = None) -> np.ndarray:
    """Midpoint-circle outline mask [nx, ny], worked in 1-based coordinates like the reference."""
    arc = min(max(2 * math.pi if arcAngle is None else arcAngle, 0.0), 2 * math.pi)
    r = int(math.copysign(math.floor(abs(radius) + 0.5), radius))  # Swift .rounded(): half away from 0
    cx1 = (_default_center(nx) if cx is None else cx) + 1
    cy1 = (_default_center(ny) if cy is None else cy) + 1
    circle = np.zeros(nx * ny, dtype=np.float32)

    def put(px: int, py: int) -> None:
        if not (math.atan2(float(px - cx1), float(py - cy1)) + math.pi <= arc):
            return
        if not (1 <= px <= nx and 1 <= py <= ny):
            return
        circle[(px - 1) * ny + (py - 1)] = 1.0

    x, y, d = 0, r, 1 - r
    put(cx1, cy1 - y)
    put(cx1, cy1 + y)
    put(cx1 + y, cy1)
    put(cx1 - y, cy1)
    while x < (y - 1):
        x += 1
        if d < 0:
            d += 2 * x + 1
        else:
            y -= 1
            d += 2 * (x - y + 1)
        px = [x + cx1, y + cx1, y + cx1, x + cx1, -x + cx1, -y + cx1, -y + cx1, -x + cx1]
        py = [y + cy1, x + cy1, -x + cy1, -y + cy1, -y + cy1, -x + cy1, x + cy1, y + cy1]
        for i in range(8):
            put(px[i], py[i])
    return circle.reshape(nx, ny)


def makeCartCircle(radius: float, numPoints: int, center: tuple[float, float] = (0.0, 0.0),
                   arcAngle: float = 2 * math.pi) -> np.ndarray:
    """Cartesian points [2, numPoints] (row 0 = x, row 1 = y) evenly spaced on a circle/arc."""
    if numPoints <= 0:
        raise ValueError("numPoints must be positive")
    full = arcAngle == 2 * math.pi
    n_steps = float(numPoints if full else numPoints - 1)
    data = np.zeros(2 * numPoints, dtype=np.float32)
    for i in range(numPoints):
        angle = float(i) * arcAngle / n_steps + math.pi / 2
        data[i] = np.float32(radius * math.cos(angle) + center[0])
        data[numPoints + i] = np.float32(radius * math.sin(-angle) + center[1])
    return data.reshape(2, numPoints)


def gaussian(x, magnitude: float | None = None, mean: float = 0.0, variance: float = 1.0) -> list[float]:
    mag = magnitude if magnitude is not None else 1.0 / math.sqrt(2 * math.pi * variance)
    return [mag * math.exp(-(v - mean) * (v - mean) / (2 * variance)) for v in x]


def toneBurst(sampleFreq: float, signalFreq: float, numCycles: float, envelope: str = "gaussian") -> np.ndarray:
    """Gaussian-enveloped (or rectangular) sine burst, float64 samples."""
    dt = 1.0 / sampleFreq
    tone_length = numCycles / signalFreq
    count = int(math.floor(tone_length / dt)) + 1
    burst = [math.sin(2 * math.pi * signalFreq * float(i) * dt) for i in range(count)]
    if envelope == "rectangular":
        window = [1.0] * count
    else:
        x_lim = 3.0
        step = 2 * x_lim / float(count - 1) if count > 1 else 0.0
        xs = [-x_lim + float(i) * step for i in range(count)]
        window = gaussian(xs, magnitude=1.0, mean=0.0, variance=1.0)
    return np.array([b * w for b, w in zip(burst, window)], dtype=np.float64)
