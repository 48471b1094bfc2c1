"""Host-side mirror of k-wave-swift's public solver API, over the CUDA library's C ABI.

Same names, argument meaning and error behaviour as the Swift types (paths relative to the
k-wave-swift project):

  KWaveGrid          Sources/KWave/Grid/KWaveGrid.swift:9-142   (makeTime 112-135, setTime 138-142)
  KWaveMedium        Sources/KWave/Medium/KWaveMedium.swift:21-76, AbsorptionMode 8-17
  KWaveSource        Sources/KWave/Source/KWaveSource.swift:11-71, SourceMode 4-8
  KWaveSensor        Sources/KWave/Sensor/KWaveSensor.swift:32-62, RecordField 4-21
  SimulationOptions  Sources/KWave/Solver/KSpaceFirstOrder.swift:17-40
  SimulationOutput   Sources/KWave/Solver/KSpaceFirstOrder.swift:47-73
  kspaceFirstOrder   Sources/KWave/Solver/KSpaceFirstOrder.swift:79-107

numpy arrays stand in for MLXArray (row-major, last axis contiguous, as MLX stores them). The
reference traps on invalid input (precondition); here the same conditions raise KWaveError.
The solver always runs on the GPU through libkwave_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import abi


class KWaveError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SourceMode(enum.IntEnum):
    dirichlet = 0
    additive = 1
    additiveNoCorrection = 2


class AbsorptionMode(enum.IntEnum):
    noAbsorption = 0
    powerLaw = 1
    noDispersion = 2
    stokes = 3


class DirectivityPattern(enum.IntEnum):
    pressure = 0
    gradient = 1


class RecordField(enum.IntFlag):
    p = 1 << 0
    pMax = 1 << 1
    pMin = 1 << 2
    pRms = 1 << 3
    pFinal = 1 << 4
    ux = 1 << 5
    uy = 1 << 6
    uz = 1 << 7
    uMax = 1 << 8
    uRms = 1 << 9
    uFinal = 1 << 10
    iAvg = 1 << 11
    iMax = 1 << 12


class DeviceKind(enum.Enum):
    gpu = "gpu"
    cpu = "cpu"
    cuda = "cuda"


def _fft_freq(n: int, d: float) -> np.ndarray:
    # Support.swift:6-14
    val = 1.0 / (n * d)
    out = np.zeros(n)
    cutoff = (n - 1) // 2 + 1
    out[:cutoff] = np.arange(cutoff) * val
    out[cutoff:] = np.arange(-(n // 2), -(n // 2) + (n - cutoff)) * val
    return out


def wavenumberVector(n: int, d: float) -> np.ndarray:
    return 2.0 * math.pi * _fft_freq(n, d)


class KWaveGrid:
    """Computational grid; unused sizes are 1 (KWaveGrid.swift:9-101)."""

    def __init__(self, nx: int, dx: float, ny: Optional[int] = None, dy: Optional[float] = None,
                 nz: Optional[int] = None, dz: Optional[float] = None):
        if ny is None:
            self.dim = 1
        elif nz is None:
            self.dim = 2
        else:
            self.dim = 3
        self.nx, self.dx = int(nx), float(dx)
        self.ny, self.dy = (int(ny), float(dy)) if ny is not None else (1, 1.0)
        self.nz, self.dz = (int(nz), float(dz)) if nz is not None else (1, 1.0)
        self.kxVec = wavenumberVector(self.nx, self.dx)
        self.kyVec = wavenumberVector(self.ny, self.dy)
        self.kzVec = wavenumberVector(self.nz, self.dz)
        self.dt = 0.0
        self.nt = 0

    @property
    def spacing(self) -> list[float]:
        return [self.dx, self.dy, self.dz][: self.dim]

    @property
    def size(self) -> list[int]:
        return [self.nx, self.ny, self.nz][: self.dim]

    @property
    def shape(self) -> tuple[int, ...]:
        return tuple(self.size)

    @property
    def totalGridPoints(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def tArray(self) -> np.ndarray:
        return np.arange(self.nt) * self.dt

    def makeTime(self, soundSpeedMax: float, soundSpeedMin: Optional[float] = None,
                 cfl: float = 0.3, tEnd: Optional[float] = None) -> None:
        """dt = cfl * min(spacing) / c_max; nt = floor(tEnd / dt) + 1 (KWaveGrid.swift:112-135)."""
        c_min = soundSpeedMin if soundSpeedMin is not None else soundSpeedMax
        dx_min = min(self.spacing)
        step = cfl * dx_min / soundSpeedMax
        if tEnd is not None:
            end = tEnd
        else:
            acc = 0.0
            for n, d in zip(self.size, self.spacing):
                extent = float(n) * d
                acc = acc + extent * extent
            end = math.sqrt(acc) / c_min
        self.dt = step
        self.nt = int(math.floor(end / step)) + 1

    def setTime(self, nt: int, dt: float) -> None:
        self.dt = float(dt)
        self.nt = int(nt)


@dataclass
class KWaveMedium:
    soundSpeed: object
    density: object
    alphaCoeff: object = None
    alphaPower: Optional[float] = None
    alphaMode: AbsorptionMode = AbsorptionMode.noAbsorption
    bOnA: object = None

    @property
    def isHomogeneous(self) -> bool:
        return np.size(self.soundSpeed) == 1 and np.size(self.density) == 1


@dataclass
class KWaveSource:
    p0: object = None
    pMask: object = None
    p: object = None
    pMode: SourceMode = SourceMode.additive
    uMask: object = None
    ux: object = None
    uy: object = None
    uz: object = None
    uMode: SourceMode = SourceMode.additive


@dataclass
class KWaveSensor:
    mask: object = None
    record: RecordField = RecordField.p
    timeReversalBoundaryData: object = None
    directivityAngle: object = None
    directivitySize: Optional[float] = None
    directivityPattern: DirectivityPattern = DirectivityPattern.pressure


@dataclass
class SimulationOptions:
    pmlSize: int = 20
    pmlAlpha: float = 2.0
    smoothP0: bool = True
    smoothC0: bool = False
    smoothRho0: bool = False
    device: DeviceKind = DeviceKind.cuda
    progress: Optional[Callable[[int, int], None]] = None
    fieldMonitor: Optional[Callable[[int, np.ndarray], None]] = None
    fieldMonitorInterval: int = 1
    cRef: Optional[float] = None      # None: max(c0), as the reference


@dataclass
class SimulationOutput:
    p: Optional[np.ndarray] = None
    pMax: Optional[np.ndarray] = None
    pMin: Optional[np.ndarray] = None
    pRms: Optional[np.ndarray] = None
    pFinal: Optional[np.ndarray] = None
    ux: Optional[np.ndarray] = None
    uy: Optional[np.ndarray] = None
    uz: Optional[np.ndarray] = None
    uxMax: Optional[np.ndarray] = None
    uyMax: Optional[np.ndarray] = None
    uzMax: Optional[np.ndarray] = None
    uxRms: Optional[np.ndarray] = None
    uyRms: Optional[np.ndarray] = None
    uzRms: Optional[np.ndarray] = None
    uxFinal: Optional[np.ndarray] = None
    uyFinal: Optional[np.ndarray] = None
    uzFinal: Optional[np.ndarray] = None
    ixAvg: Optional[np.ndarray] = None
    iyAvg: Optional[np.ndarray] = None
    izAvg: Optional[np.ndarray] = None


# ------------------------------------------------------------------------------------------
# Descriptor construction (shared by the CUDA binding and the test oracle binding)
# ------------------------------------------------------------------------------------------

def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class DescBuilder:
    """Flattens the mirror structs into one kw_sim_desc, keeping the host arrays alive."""

    def __init__(self, grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                 sensor: KWaveSensor, options: Optional[SimulationOptions] = None, axisymmetric: bool = False):
        options = options or SimulationOptions()
        self.keep: list[np.ndarray] = []
        self.grid = grid
        self.medium, self.source, self.sensor, self.options = medium, source, sensor, options
        shape = grid.shape
        N = grid.totalGridPoints
        d = abi.kw_sim_desc()
        d.abi_version = abi.KW_ABI_VERSION
        d.dim = grid.dim
        d.nx, d.ny, d.nz = grid.nx, grid.ny, grid.nz
        d.dx, d.dy, d.dz = grid.dx, grid.dy, grid.dz
        d.dt, d.nt = grid.dt, grid.nt
        d.axisymmetric = int(bool(axisymmetric))
        d.pml_size = int(options.pmlSize)
        d.pml_alpha = float(options.pmlAlpha)
        d.smooth_p0 = int(bool(options.smoothP0))
        d.smooth_c0 = int(bool(options.smoothC0))
        d.smooth_rho0 = int(bool(options.smoothRho0))
        d.c_ref = math.nan if options.cRef is None else float(options.cRef)

        def scalar_or_grid(x, name, required):
            if x is None:
                if required:
                    raise KWaveError(abi.KW_ERR_INVALID, f"{name} is required")
                return abi.kw_array()
            a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
            if a.size != 1 and tuple(a.shape) != shape:
                raise KWaveError(abi.KW_ERR_INVALID, f"{name} must be scalar or {list(shape)}")
            a = a.reshape(-1)
            self.keep.append(a)
            return abi.kw_array(_fptr(a), a.size)

        def grid_array(x, name):
            if x is None:
                return None
            a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
            if a.size != N:
                raise KWaveError(abi.KW_ERR_INVALID, f"{name} must have the grid shape {list(shape)}")
            a = a.reshape(-1)
            self.keep.append(a)
            return _fptr(a)

        def signal(x):
            if x is None:
                return abi.kw_signal()
            a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
            if a.ndim <= 1:
                a = a.reshape(1, -1)
            rows, length = a.shape[0], a.shape[1]
            a = a.reshape(-1)
            self.keep.append(a)
            return abi.kw_signal(_fptr(a), rows, length)

        d.sound_speed = scalar_or_grid(medium.soundSpeed, "soundSpeed", True)
        d.density = scalar_or_grid(medium.density, "density", True)
        d.alpha_coeff = scalar_or_grid(medium.alphaCoeff, "alphaCoeff", False)
        d.alpha_power = math.nan if medium.alphaPower is None else float(medium.alphaPower)
        d.alpha_mode = int(medium.alphaMode)
        d.b_on_a = scalar_or_grid(medium.bOnA, "bOnA", False)

        d.p0 = grid_array(source.p0, "p0")
        d.p_mask = grid_array(source.pMask, "pMask")
        d.p = signal(source.p)
        d.p_mode = int(source.pMode)
        d.u_mask = grid_array(source.uMask, "uMask")
        d.ux, d.uy, d.uz = signal(source.ux), signal(source.uy), signal(source.uz)
        d.u_mode = int(source.uMode)

        d.record = int(sensor.record)
        d.sensor_kind = abi.KW_SENSOR_NONE
        if sensor.mask is not None:
            m = np.asarray(sensor.mask, dtype=np.float32)
            if m.ndim == 2 and m.shape[0] == grid.dim:     # Recording.swift:51 Cartesian detection
                m = np.ascontiguousarray(m)
                d.sensor_kind = abi.KW_SENSOR_CARTESIAN
                d.sensor_points = m.shape[1]
                flat = m.reshape(-1)
                self.keep.append(flat)
                d.sensor_mask = _fptr(flat)
            else:
                d.sensor_kind = abi.KW_SENSOR_BINARY
                d.sensor_mask = grid_array(m, "sensor.mask")
        d.directivity_angle = grid_array(sensor.directivityAngle, "directivityAngle") \
            if sensor.directivityAngle is not None else None
        d.directivity_size = math.nan if sensor.directivitySize is None else float(sensor.directivitySize)
        d.directivity_pattern = int(sensor.directivityPattern)
        self.desc = d
        self.shape = shape


def output_shape(field_name: str, shape: tuple, n_sensor: int, steps: int, count: int) -> tuple:
    if field_name in ("p", "ux", "uy", "uz"):
        return (n_sensor, steps)
    if field_name.endswith("Final"):
        return tuple(shape)
    return (count,)


# ------------------------------------------------------------------------------------------
# The CUDA solver
# ------------------------------------------------------------------------------------------

def kspaceFirstOrder(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                     sensor: KWaveSensor, options: Optional[SimulationOptions] = None) -> SimulationOutput:
    """k-space pseudospectral fluid solver (1D/2D/3D) on the GPU (KSpaceFirstOrder.swift:79-107)."""
    from .runtime import Context

    options = options or SimulationOptions()
    if options.device == DeviceKind.cpu:
        raise KWaveError(abi.KW_ERR_UNSUPPORTED, "this build runs on CUDA devices only")
    if grid.dim not in (1, 2, 3):
        raise KWaveError(abi.KW_ERR_INVALID, f"kspaceFirstOrder: dim {grid.dim} not yet implemented")
    with Context.default() as ctx:
        sim = ctx.create_sim(DescBuilder(grid, medium, source, sensor, options))
        try:
            sim.run(progress=options.progress, monitor=options.fieldMonitor,
                    monitor_interval=options.fieldMonitorInterval)
            return sim.outputs()
        finally:
            sim.close()


def kspaceFirstOrderAS(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                       sensor: KWaveSensor, options: Optional[SimulationOptions] = None) -> SimulationOutput:
    """Axisymmetric k-space solver on the GPU (KSpaceFirstOrderAS.swift:19-309): a 2D grid with x
    axial and y radial (r >= 0); p0 and pressure / velocity sources, Stokes absorption, B/A;
    returns p and pFinal."""
    from .runtime import Context

    options = options or SimulationOptions()
    if options.device == DeviceKind.cpu:
        raise KWaveError(abi.KW_ERR_UNSUPPORTED, "this build runs on CUDA devices only")
    if grid.dim != 2:
        raise KWaveError(abi.KW_ERR_INVALID, "axisymmetric solver requires a 2D grid (x axial, y radial)")
    with Context.default() as ctx:
        sim = ctx.create_sim(DescBuilder(grid, medium, source, sensor, options, axisymmetric=True))
        try:
            sim.run(progress=options.progress, monitor=options.fieldMonitor,
                    monitor_interval=options.fieldMonitorInterval)
            return sim.outputs()
        finally:
            sim.close()


@dataclass
class AdjointOutput:
    misfit: float
    gradSoundSpeed: Optional[np.ndarray]
    gradP0: Optional[np.ndarray]
    gradRho0: Optional[np.ndarray]
    forwardMs: float
    reverseMs: float
    checkpointInterval: int
    checkpoints: int


def kspaceFirstOrderAdjoint(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource, sensor: KWaveSensor,
                            data: np.ndarray, options: Optional[SimulationOptions] = None,
                            gradP0: bool = False, checkpointPolicy: int = abi.KW_CHECKPOINT_SQRT,
                            checkpointInterval: int = 0, memoryBudget: float = 0.0,
                            gradRho0: bool = False) -> AdjointOutput:
    """Misfit 1/2 sum (p_sensor - data)^2 of the forward kspaceFirstOrder run and its gradients
    with respect to the sound speed (and the initial pressure, and the density), by the discrete
    adjoint (kw_adjoint_run). `data` has the layout of the p output, [n_sensor, nt]."""
    from .runtime import Context

    options = options or SimulationOptions()
    with Context.default() as ctx:
        r = ctx.adjoint(DescBuilder(grid, medium, source, sensor, options), data, True, gradP0,
                        checkpointPolicy, checkpointInterval, memoryBudget, grad_rho0=gradRho0)
    return AdjointOutput(r["misfit"], r["grad_c0"], r["grad_p0"], r["grad_rho0"], r["forward_ms"], r["reverse_ms"],
                         r["interval"], r["checkpoints"])


def timeReversal(grid: KWaveGrid, medium: KWaveMedium, sensor: KWaveSensor, recordedPressure: np.ndarray,
                 compensationFactor: float = 2.0, options: Optional[SimulationOptions] = None) -> np.ndarray:
    """Time-reversal reconstruction (Sources/KWave/Reconstruction/TimeReversal.swift:20-51): the
    recorded sensor pressure [n_sensor, nt], flipped in time, is re-injected as a Dirichlet
    pressure source on the sensor mask; the solver runs forward over the whole grid and the final
    pressure, scaled by `compensationFactor` and clipped at zero, is the estimate of p0."""
    if sensor.mask is None:
        raise KWaveError(abi.KW_ERR_INVALID, "time reversal requires sensor.mask")
    if grid.nt <= 0:
        raise KWaveError(abi.KW_ERR_INVALID, "set grid time (makeTime/setTime) before time reversal")
    rec = np.asarray(recordedPressure, np.float32)
    if rec.ndim != 2:
        raise KWaveError(abi.KW_ERR_INVALID, "recordedPressure must be [numSensorPoints, nt]")
    source = KWaveSource(pMask=np.asarray(sensor.mask, np.float32), p=np.ascontiguousarray(rec[:, ::-1]),
                         pMode=SourceMode.dirichlet)
    out = kspaceFirstOrder(grid, medium, source, KWaveSensor(), options)
    p0 = out.pFinal * np.float32(compensationFactor)
    return np.maximum(p0, np.float32(0))

