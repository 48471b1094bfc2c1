"""CPU tests of the FP64 oracle: known answers from the reference's own tests, self-consistency
(symmetry) tests from Tests/KWaveTests/SolverTests.swift, and agreement with the independent
numpy restatement stored in tests/golden/."""
import math

import numpy as np
import pytest

import oracle
from cases import GOLDEN_AS_CASES, GOLDEN_CASES, builder_from_case, load_golden, rel_l2, rel_max
from kwave import (DescBuilder, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, RecordField,
                   SimulationOptions, makeCircle, makeDisc, toneBurst)


@pytest.mark.parametrize("name", GOLDEN_CASES + GOLDEN_AS_CASES)
def test_oracle_matches_numpy_restatement(name):
    case, ref = load_golden(name)
    out, _ = oracle.run(builder_from_case(case))
    for k, v in ref.items():
        assert out[k] is not None, k
        assert out[k].shape == v.shape, (k, out[k].shape, v.shape)
        assert rel_max(out[k], v) < 1e-9, (k, rel_max(out[k], v))
    for k, v in out.items():
        if v is not None:
            assert k in ref, f"oracle produced {k} the restatement did not"


def test_fft_matches_numpy():
    rng = np.random.default_rng(1)
    for n in (1, 2, 3, 5, 7, 8, 12, 24, 48, 64, 96, 101, 128, 192, 256, 384):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(oracle.fft(x), np.fft.fft(x), rtol=1e-12, atol=1e-12 * n)
        assert np.allclose(oracle.fft(x, inverse=True), np.fft.ifft(x) * n, rtol=1e-12, atol=1e-12 * n)


def test_make_time_known_answers():
    # ParityTests.swift:63 — 64x64, dx 1e-4, c 1500, cfl 0.3, default tEnd -> nt == 302
    g = KWaveGrid(64, 1e-4, 64, 1e-4)
    g.makeTime(1500.0, cfl=0.3)
    assert g.nt == 302
    # GridTests.swift:18-24 — dt = cfl*dx/c
    g = KWaveGrid(16, 1e-3, 16, 1e-3)
    g.makeTime(1500.0, cfl=0.3)
    assert abs(g.dt - 0.3 * 1e-3 / 1500) < 1e-12 and g.nt > 0
    # the 128^2 IVP workload: tEnd 4 us -> dt 2e-8, nt 201
    g = KWaveGrid(128, 1e-4, 128, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=4e-6)
    assert abs(g.dt - 2e-8) < 1e-20 and g.nt == 201


def test_wavenumbers_dc_zero():
    # GridTests.swift:8-16
    g = KWaveGrid(8, 1e-3, 4, 2e-3)
    assert g.kxVec[0] == 0 and g.totalGridPoints == 32


def test_make_circle_known_answer():
    # UtilTests.swift:8-16
    c = makeCircle(11, 11, radius=3)
    assert int(c.sum()) == 16
    for x, y in [(2, 4), (3, 3), (4, 2), (5, 8), (8, 6)]:
        assert c[x, y] == 1


def test_tone_burst_known_answer():
    # UtilTests.swift:199-208
    b = toneBurst(10e6, 1e6, 3.0)
    assert len(b) == int(math.floor((3.0 / 1e6) / (1 / 10e6))) + 1
    mid = np.max(np.abs(b))
    assert abs(b[0]) < mid and abs(b[-1]) < mid


def test_db2neper_roundtrip():
    # UtilTests.swift:139-143
    np_ = oracle.db2neper(0.75, 1.5)
    back = 20 * math.log10(math.e) * np_ * (2 * math.pi * 1e6) ** 1.5 / 100
    assert abs(back - 0.75) < 1e-12


def test_pml_profile_shape():
    p = oracle.pml_profile(64, 1e-4, 2e-8, 1500.0, 20, 2.0, False)
    ps = oracle.pml_profile(64, 1e-4, 2e-8, 1500.0, 20, 2.0, True)
    assert np.all(p[20:44] == 1.0) and np.all(ps[20:44] == 1.0)
    assert p[0] < p[19] < 1.0 and ps[63] < ps[44] < 1.0
    # PML.swift:21-22: left and right are computed independently (staggered is not a mirror)
    assert not np.allclose(ps[:20], ps[44:][::-1])


def crefl(a, axis):
    return np.roll(np.flip(a, axis=axis), 1, axis=axis)


def test_oracle_1d_symmetric_ivp():
    # SolverTests.swift:18-47
    n = 64
    g = KWaveGrid(n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=4e-7)
    p0 = np.zeros(n, np.float32)
    p0[n // 2 - 3:n // 2 + 4] = 1
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=p0), KWaveSensor())
    out, _ = oracle.run(b)
    pf = out["pFinal"]
    m = np.max(np.abs(pf))
    assert np.isfinite(m) and m > 0
    assert np.max(np.abs(pf - crefl(pf, 0))) / m < 1e-3


def test_oracle_2d_disc_symmetric():
    # SolverTests.swift:78-103
    n = 64
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=3e-7)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(n, n, radius=5)), KWaveSensor())
    out, _ = oracle.run(b)
    pf = out["pFinal"]
    m = np.max(np.abs(pf))
    assert m > 0
    assert np.max(np.abs(pf - crefl(pf, 0))) / m < 1e-3
    assert np.max(np.abs(pf - crefl(pf, 1))) / m < 1e-3


def test_oracle_line_sensor_shape():
    # SolverTests.swift:106-126
    n = 48
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=4e-6)
    mask = np.zeros((n, n), np.float32)
    mask[8, :] = 1
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(n, n, radius=4)),
                    KWaveSensor(mask=mask))
    out, _ = oracle.run(b)
    assert out["p"].shape == (n, g.nt) and np.all(np.isfinite(out["p"]))


def test_oracle_1d_time_varying_source_shape():
    # SolverTests.swift:51-74
    n = 96
    g = KWaveGrid(n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=5e-6)
    m = np.zeros(n, np.float32)
    m[16] = 1
    s = np.zeros(n, np.float32)
    s[64] = 1
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0),
                    KWaveSource(pMask=m, p=toneBurst(1 / g.dt, 1e6, 3).astype(np.float32)),
                    KWaveSensor(mask=s))
    out, _ = oracle.run(b)
    assert out["p"].shape == (1, g.nt)
    assert np.max(np.abs(out["p"])) > 0


def test_smoothing_window_2d_vs_3d_convention():
    # Filters.swift: 2D fills out[i] = win[(i+s)%n]; 3D fills out[(i+s)%n] = win[i] (odd sizes differ)
    w2 = oracle.smoothing_window((7, 8))
    assert w2.shape == (7, 8) and np.all(w2 >= 0) and np.max(w2) <= 1.0 + 1e-12
    w3 = oracle.smoothing_window((8, 8, 8))
    assert abs(w3[0, 0, 0] - 1.0) < 1e-12


def test_invalid_descriptors_rejected():
    g = KWaveGrid(16, 1e-4, 16, 1e-4)
    g.makeTime(1500.0)
    with pytest.raises(oracle.OracleError):
        oracle.run(DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(), KWaveSensor()))
    g2 = KWaveGrid(16, 1e-4, 16, 1e-4)   # no makeTime
    with pytest.raises(oracle.OracleError):
        oracle.run(DescBuilder(g2, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(16, 16, radius=2)), KWaveSensor()))
