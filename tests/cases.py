"""Shared helpers: build kwave mirror objects from golden-case dicts and compare outputs."""
from __future__ import annotations

import os

import numpy as np

from kwave import (AbsorptionMode, DescBuilder, DirectivityPattern, KWaveGrid, KWaveMedium, KWaveSensor,
                   KWaveSource, RecordField, SimulationOptions, SourceMode)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = ["1d_source_hetero", "2d_ivp", "2d_hetero_abs_nl", "2d_stokes_nc", "3d_hetero_src",
                "2d_directivity_pressure", "2d_directivity_gradient"]
# axisymmetric (kspaceFirstOrderAS) golden cases
GOLDEN_AS_CASES = ["as_ivp", "as_add", "as_dir", "as_stokes", "as_nl", "as_uxs", "as_uys", "as_hetero"]


def load_golden(name: str):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    case, src, out = {}, {}, {}
    for k in z.files:
        v = z[k]
        if k.startswith("in_"):
            case[k[3:]] = v
        elif k.startswith("src_"):
            src[k[4:]] = v
        else:
            out[k[4:]] = v
    case["source"] = src
    return case, out


def builder_from_case(case) -> DescBuilder:
    dim = int(case["dim"])
    shape = [int(v) for v in case["shape"]]
    sp = [float(v) for v in case["spacing"]]
    args = []
    for a in range(dim):
        args += [shape[a], sp[a]]
    grid = KWaveGrid(*args)
    grid.setTime(int(case["nt"]), float(case["dt"]))

    def opt(k):
        return case[k] if k in case else None

    medium = KWaveMedium(soundSpeed=case["c0"], density=case["rho0"], alphaCoeff=opt("alpha_coeff"),
                         alphaPower=float(case["alpha_power"]) if "alpha_power" in case else None,
                         alphaMode=AbsorptionMode(int(case.get("alpha_mode", 0))), bOnA=opt("b_on_a"))
    s = case["source"]
    source = KWaveSource(p0=s.get("p0"), pMask=s.get("p_mask"), p=s.get("p"),
                         pMode=SourceMode(int(s.get("p_mode", 1))), uMask=s.get("u_mask"),
                         ux=s.get("ux"), uy=s.get("uy"), uz=s.get("uz"),
                         uMode=SourceMode(int(s.get("u_mode", 1))))
    sensor = KWaveSensor(mask=case.get("sensor_mask"), record=RecordField(int(case["record"])))
    if "directivity_angle" in case:
        sensor.directivityAngle = case["directivity_angle"]
        sensor.directivitySize = float(case["directivity_size"])
        sensor.directivityPattern = DirectivityPattern(int(case["directivity_pattern"]))
    options = SimulationOptions(pmlSize=int(case["pml_size"]), pmlAlpha=float(case.get("pml_alpha", 2.0)),
                                smoothP0=bool(case.get("smooth_p0", True)),
                                smoothC0=bool(case.get("smooth_c0", False)),
                                smoothRho0=bool(case.get("smooth_rho0", False)))
    return DescBuilder(grid, medium, source, sensor, options, axisymmetric=bool(case.get("axisymmetric", 0)))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt(np.sum(b * b))
    return float(np.sqrt(np.sum((a - b) ** 2)) / den) if den > 0 else float(np.sqrt(np.sum(a * a)))


def rel_max(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a)))
