"""kwave — B200 (sm_100a) k-space pseudospectral fluid solver with k-wave-swift's API.

The solver runs in libkwave_cuda.so (hand-written CUDA for sm_100a behind a C ABI,
include/kwave_cuda.h). This package mirrors the reference's Swift API over that ABI.
"""
from .abi import FIELDS
from .api import (AbsorptionMode, AdjointOutput, DescBuilder, DeviceKind, DirectivityPattern, KWaveError,
                  KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, RecordField,
                  SimulationOptions, SimulationOutput, SourceMode, kspaceFirstOrder,
                  kspaceFirstOrderAdjoint, kspaceFirstOrderAS, timeReversal, wavenumberVector)
from .shapes import gaussian, makeBall, makeCartCircle, makeCircle, makeDisc, toneBurst

__all__ = [
    "AbsorptionMode", "AdjointOutput", "DescBuilder", "DeviceKind", "DirectivityPattern", "FIELDS", "KWaveError",
    "KWaveGrid", "KWaveMedium", "KWaveSensor", "KWaveSource", "RecordField", "SimulationOptions",
    "SimulationOutput", "SourceMode", "gaussian", "kspaceFirstOrder", "kspaceFirstOrderAS", "kspaceFirstOrderAdjoint",
    "makeBall",
    "makeCartCircle", "makeCircle", "makeDisc", "timeReversal", "toneBurst", "wavenumberVector",
]
