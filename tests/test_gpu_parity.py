"""GPU parity: the CUDA library (through its C ABI) against the FP64 oracle / golden fixtures.

Tolerances (FP32 device arithmetic vs FP64 oracle): relative L2 <= 1e-4 on pressure time series
and final fields; relative L2 <= 1e-3 on aggregates derived from sampled series and intensity.
Sensor counts and row ordering must match exactly.
"""
import numpy as np
import pytest

import oracle
from cases import GOLDEN_CASES, builder_from_case, load_golden, rel_l2, rel_max
from kwave import (DescBuilder, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, RecordField,
                   SimulationOptions, SourceMode, makeBall, makeCartCircle, makeCircle, makeDisc,
                   toneBurst)
from kwave.runtime import Context

pytestmark = pytest.mark.gpu

TIGHT = {"p", "pFinal", "ux", "uy", "uz", "uxFinal", "uyFinal", "uzFinal"}


def run_gpu(builder):
    ctx = Context.default()
    sim = ctx.create_sim(builder)
    try:
        sim.run()
        return {k: v for k, v in vars(sim.outputs()).items()}
    finally:
        sim.close()


def compare(out, ref, tight=1e-4, loose=1e-3):
    for k, v in ref.items():
        if v is None:
            continue
        assert out.get(k) is not None, f"missing output {k}"
        assert out[k].shape == v.shape, (k, out[k].shape, v.shape)
        e = rel_l2(out[k], v)
        tol = tight if k in TIGHT else loose
        assert e < tol, f"{k}: rel L2 {e:.3e} >= {tol}"
    for k, v in out.items():
        if v is not None:
            assert ref.get(k) is not None, f"unexpected output {k}"


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_case(name):
    case, ref = load_golden(name)
    # the gradient directivity pattern is odd in k, so Re F^-1 keeps only the self-conjugate
    # (Nyquist) bins: a signal ~1e-3 of the pressure pattern's, checked at 1e-3 as
    # ParityDirectivityTests.swift:78-80 does
    compare(run_gpu(builder_from_case(case)), ref, tight=1e-3 if name == "2d_directivity_gradient" else 1e-4)


def c1_builder(nt=None):
    n = 128
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=4e-6)
    if nt is not None:
        g.setTime(nt, g.dt)
    src = KWaveSource(p0=makeDisc(n, n, radius=5) * 1.0)
    sen = KWaveSensor(mask=makeCircle(n, n, radius=40), record=RecordField.p | RecordField.pFinal | RecordField.pMax)
    return DescBuilder(g, KWaveMedium(1500.0, 1000.0), src, sen, SimulationOptions(pmlSize=20, smoothP0=True))


def test_c1_2d_ivp_vs_oracle():
    b = c1_builder()
    assert b.grid.nt == 201
    ref, _ = oracle.run(b)
    out = run_gpu(b)
    assert out["p"].shape == (224, 201)
    compare(out, ref)


def test_3d_hetero_nonlinear_absorbing_source_vs_oracle():
    rng = np.random.default_rng(7)
    n = 40
    dx = 1e-4
    c = np.full((n, n, n), 1500, np.float32)
    rho = np.full((n, n, n), 1000, np.float32)
    for _ in range(3):
        r = rng.integers(3, 7)
        cx, cy, cz = rng.integers(10, 30, size=3)
        m = makeBall(n, n, n, cx, cy, cz, r) > 0
        c[m] = rng.uniform(1400, 1650)
        rho[m] = rng.uniform(900, 1100)
    g = KWaveGrid(n, dx, n, dx, n, dx)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(60, g.dt)
    pm = np.zeros((n, n, n), np.float32)
    pm[14:26, 14:26, 8] = 1
    sig = (toneBurst(1 / g.dt, 1e6, 3) * 1e6).astype(np.float32)
    sm = np.zeros((n, n, n), np.float32)
    sm[:, :, 20] = 1
    med = KWaveMedium(c, rho, alphaCoeff=0.75, alphaPower=1.5, alphaMode=1, bOnA=6.0)
    b = DescBuilder(g, med, KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                    KWaveSensor(mask=sm, record=RecordField.p | RecordField.pMax), SimulationOptions(pmlSize=8))
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)


def crefl(a, axis):
    return np.roll(np.flip(a, axis=axis), 1, axis=axis)


def test_gpu_2d_disc_symmetric():
    # SolverTests.swift:78-103 on the device
    n = 64
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=3e-7)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(n, n, radius=5)), KWaveSensor())
    pf = run_gpu(b)["pFinal"]
    m = np.max(np.abs(pf))
    assert m > 0 and np.max(np.abs(pf - crefl(pf, 0))) / m < 1e-3 and np.max(np.abs(pf - crefl(pf, 1))) / m < 1e-3


def test_gpu_3d_ivp_matches_oracle():
    # GPUSmokeTests.swift:77-89 shape: 24^3 ball r=3, tEnd 3e-7
    n = 24
    g = KWaveGrid(n, 1e-4, n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3, tEnd=3e-7)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeBall(n, n, n, radius=3)), KWaveSensor())
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)


def test_odd_sizes_and_generic_radix():
    # odd contiguous axis (R2C without the packed path) and a prime-factor length (generic radix)
    g = KWaveGrid(34, 1e-4, 27, 1e-4)
    g.setTime(30, 2e-8)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(34, 27, radius=3)),
                    KWaveSensor(mask=makeCircle(34, 27, radius=8), record=RecordField.p), SimulationOptions(pmlSize=5))
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)
    g = KWaveGrid(22, 1e-4, 26, 1e-4, 21, 1e-4)
    g.setTime(20, 2e-8)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeBall(22, 26, 21, radius=3)), KWaveSensor(),
                    SimulationOptions(pmlSize=4))
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)


def _reg_case(shape, seed, pml):
    """Heterogeneous nonlinear power-law case with an additive plane source, for the kernel lengths
    of the register-resident passes (radix-12 and long power-of-two lines)."""
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
    sl = tuple([slice(pml + 1, n - pml - 1) for n in shape[:-1]] + [pml + 2])
    pm[sl] = 1
    sig = (toneBurst(1 / g.dt, 2e6, 2) * 1e5).astype(np.float32)
    sm = np.zeros(shape, np.float32)
    sm[tuple([slice(None)] * (dim - 1) + [pml + 8])] = 1   # within reach of the source in 40 steps
    med = KWaveMedium(c, rho, alphaCoeff=0.5, alphaPower=1.5, alphaMode=1, bOnA=5.0)
    return DescBuilder(g, med, KWaveSource(pMask=pm, p=sig, pMode=SourceMode.additive),
                       KWaveSensor(mask=sm, record=RecordField.p | RecordField.pFinal), SimulationOptions(pmlSize=pml))


@pytest.mark.parametrize("shape", [(96, 192), (384, 48), (1024, 64), (32, 4096), (48, 24, 96), (24, 192, 40),
                                   (16, 32, 32)])
def test_register_plan_lengths(shape):
    # radix-12 plans (24 ... 768), long rows (C = 4096: half length 2048) and long operator
    # columns (1024); in 3D the TMA-fed in-place pass runs along B
    b = _reg_case(shape, sum(shape), 6)
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)


@pytest.mark.parametrize("cola", ["1", "3"])
@pytest.mark.parametrize("shape", [(96, 192), (1024, 64), (48, 24, 96), (24, 192, 40), (16, 32, 32), (20, 384, 16),
                                   (16, 512, 24)])
def test_double_buffered_column_passes(shape, cola, monkeypatch):
    # the double-buffered register column kernel for the operator pass (KW_COLA=1) and also for the
    # in-place passes up to 256 points (KW_COLA=3); in 3D along B lengths above 256 take it anyway
    monkeypatch.setenv("KW_COLA", cola)
    b = _reg_case(shape, sum(shape) // 2, 6)
    ref, _ = oracle.run(b)
    compare(run_gpu(b), ref)


def _plane_case(shape, seed):
    """3D heterogeneous nonlinear power-law IVP (a p0 ball off centre) with a sensor plane, thin
    along A so that long B and C lines stay cheap for the oracle."""
    rng = np.random.default_rng(seed)
    c = (1500 + 60 * rng.standard_normal(shape)).astype(np.float32)
    rho = (1000 + 40 * rng.standard_normal(shape)).astype(np.float32)
    args = []
    for n in shape:
        args += [n, 1e-4]
    g = KWaveGrid(*args)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(24, g.dt)
    a, b, cc = shape
    p0 = makeBall(a, b, cc, a // 2, b // 3, cc // 2 + 3, 3) * 1e4
    sm = np.zeros(shape, np.float32)
    sm[:, :, cc // 2] = 1
    med = KWaveMedium(c, rho, alphaCoeff=0.5, alphaPower=1.5, alphaMode=1, bOnA=5.0)
    return DescBuilder(g, med, KWaveSource(p0=p0), KWaveSensor(mask=sm, record=RecordField.p | RecordField.pFinal),
                       SimulationOptions(pmlSize=4, smoothP0=False))


@pytest.mark.parametrize("plane", ["1", "0"])
@pytest.mark.parametrize("shape", [(16, 32, 32), (12, 48, 48), (12, 64, 128), (10, 128, 256), (10, 256, 256),
                                   (10, 384, 384)])
def test_plane_pass_shapes(shape, plane, monkeypatch):
    # 3D: the R2C and the forward pass along B as one cluster kernel per plane (cluster sizes 1, 2,
    # 4 and 8, the packed DC / Nyquist column) against the separate passes and the oracle
    monkeypatch.setenv("KW_PLANE", plane)
    b = _plane_case(shape, sum(shape) // 3)
    ref, _ = oracle.run(b)
    out = run_gpu(b)
    assert np.abs(ref["p"]).max() > 0
    compare(out, ref)


def test_batch_equals_individual_runs(monkeypatch):
    # bit for bit with fixed kernel variants (the autotuner may pick another radix split for the
    # batch's larger launches, whose results then differ in the last bits)
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    rng = np.random.default_rng(3)
    builders = []
    for n in (48, 64, 40):
        g = KWaveGrid(n, 1e-4, n, 1e-4)
        g.makeTime(1500.0, cfl=0.3)
        g.setTime(int(rng.integers(30, 60)), g.dt)
        sm = makeCartCircle(0.3 * n * 1e-4, 16)
        pm = np.zeros((n, n), np.float32)
        pm[10, 5:9] = 1
        src = KWaveSource(pMask=pm, p=toneBurst(1 / g.dt, 2e6, 2).astype(np.float32))
        builders.append(DescBuilder(g, KWaveMedium(1500.0, 1000.0), src, KWaveSensor(mask=sm, record=RecordField.p)))
    ctx = Context.default()
    singles = [run_gpu(b) for b in builders]
    batch = ctx.create_batch(builders)
    try:
        batch.run()
        for i, b in enumerate(builders):
            p = batch.output(i, "p", b.grid.nt, 16)
            assert np.array_equal(p, singles[i]["p"]), i
            assert np.array_equal(batch.output(i, "pFinal", b.grid.nt, 16), singles[i]["pFinal"]), i
    finally:
        batch.close()


def test_batch_with_and_without_directivity(monkeypatch):
    # the per-angle filter jobs gate themselves per simulation: a batch mixing a directivity
    # sensor, a plain sensor and a second angle set gives each simulation's own run
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    builders = [builder_from_case(load_golden(n)[0]) for n in ("2d_directivity_pressure", "2d_ivp",
                                                               "2d_directivity_gradient")]
    singles = [run_gpu(b) for b in builders]
    batch = Context.default().create_batch(builders)
    try:
        batch.run()
        for i, b in enumerate(builders):
            npts = singles[i]["p"].shape[0]
            assert np.array_equal(batch.output(i, "p", b.grid.nt, npts), singles[i]["p"]), i
    finally:
        batch.close()


def test_kspace_first_order_api_progress_and_monitor():
    from kwave import kspaceFirstOrder
    n = 32
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.setTime(12, 2e-8)
    steps, mons = [], []
    opts = SimulationOptions(pmlSize=6, progress=lambda t, nt: steps.append((t, nt)),
                             fieldMonitor=lambda t, p: mons.append((t, p.shape)), fieldMonitorInterval=5)
    out = kspaceFirstOrder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(n, n, radius=3)), KWaveSensor(), opts)
    assert out.pFinal.shape == (n, n)
    assert steps == [(t, 12) for t in range(12)]
    assert [m[0] for m in mons] == [0, 5, 10] and all(m[1] == (n, n) for m in mons)


def test_time_reversal_matches_oracle():
    # the shape of ParityTests.swift:271-329: a disc p0 radiates to a circular sensor; the recorded
    # pressure is re-injected time-reversed as a Dirichlet source; the compensated, clipped final
    # pressure is the reconstruction
    from kwave import timeReversal
    n = 64
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.makeTime(1500.0, cfl=0.3)
    med = KWaveMedium(1500.0, 1000.0)
    mask = makeCircle(n, n, radius=24)
    fwd = DescBuilder(g, med, KWaveSource(p0=makeDisc(n, n, radius=4) * 1.0),
                      KWaveSensor(mask=mask, record=RecordField.p), SimulationOptions(pmlSize=10))
    rec = run_gpu(fwd)["p"]
    mine = timeReversal(g, med, KWaveSensor(mask=mask), rec, compensationFactor=2.0,
                        options=SimulationOptions(pmlSize=10))
    tr = DescBuilder(g, med, KWaveSource(pMask=mask, p=np.ascontiguousarray(rec[:, ::-1]), pMode=SourceMode.dirichlet),
                     KWaveSensor(), SimulationOptions(pmlSize=10))
    ref = np.maximum(oracle.run(tr)[0]["pFinal"] * 2.0, 0.0)
    assert rel_l2(mine, ref) < 1e-4, rel_l2(mine, ref)
    assert rel_max(mine, ref) < 1e-4, rel_max(mine, ref)


@pytest.mark.parametrize("shape", [(256, 24, 32), (256, 96), (512, 64), (512, 512)])
def test_operator_pass_lengths_of_the_benchmarks(shape):
    # the operator column pass at the lengths the benchmarks run: along A = 256 in 3D (the 256^3
    # forward), along B = 256 and 512 in 2D (the 2D batch and the 512^2 adjoint workload);
    # heterogeneous, power law + B/A, additive source
    b = _reg_case(shape, sum(shape) + 1, 6)
    ref, _ = oracle.run(b)
    assert np.abs(ref["p"]).max() > 0
    compare(run_gpu(b), ref)


def _rowwise_order_check(out_p, ref_p):
    # every sensor row against the oracle's row of the same index: a permutation of rows fails
    # because distinct rows differ by far more than the tolerance
    scale = np.abs(ref_p).max()
    assert scale > 0
    err = np.abs(out_p.astype(np.float64) - ref_p).max(axis=1) / scale
    assert err.max() < 1e-4, err.max()
    # for the check to pin the order, every row the wave has reached (peak above 1 % of the
    # largest) must differ from every other row by far more than the tolerance; rows it has not
    # reached are all ~0 and interchangeable
    live = np.abs(ref_p).max(axis=1) > 1e-2 * scale
    idx = np.nonzero(live)[0]
    assert len(idx) >= len(ref_p) // 2, (len(idx), len(ref_p))
    d = np.abs(ref_p[idx][:, None, :] - ref_p[None, :, :]).max(axis=2) / scale
    d[np.arange(len(idx)), idx] = np.inf
    assert d.min() > 2e-3, d.min()


@pytest.mark.parametrize("shape", [(60, 52), (28, 34, 30)])
def test_binary_sensor_order_asymmetric(shape):
    # flatNonzeroIndices order (KSpaceFirstOrder.swift:778-782): rows in ascending row-major flat
    # index; random mask, random heterogeneous medium, off-centre source
    rng = np.random.default_rng(sum(shape))
    dx = 1e-4
    c = (1500 + 80 * rng.standard_normal(shape)).astype(np.float32)
    rho = (1000 + 50 * rng.standard_normal(shape)).astype(np.float32)
    args = []
    for n in shape:
        args += [n, dx]
    g = KWaveGrid(*args)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(70, g.dt)
    p0 = np.zeros(shape, np.float32)
    p0[tuple(slice(n // 3, n // 3 + 3) for n in shape)] = 1e3
    inner = np.zeros(shape, bool)
    inner[tuple(slice(6, n - 6) for n in shape)] = True
    mask = ((rng.random(shape) < (60 / inner.sum())) & inner).astype(np.float32)
    b = DescBuilder(g, KWaveMedium(c, rho), KWaveSource(p0=p0), KWaveSensor(mask=mask, record=RecordField.p),
                    SimulationOptions(pmlSize=5, smoothP0=False))
    ref, _ = oracle.run(b)
    out = run_gpu(b)
    assert out["p"].shape == (int(mask.sum()), 70)
    _rowwise_order_check(out["p"], ref["p"])


def test_cartesian_sensor_order_random_points():
    # Cartesian sensor rows follow the input column order (Recording.swift:51-97): random
    # off-grid points in random order, multilinear interpolation
    rng = np.random.default_rng(11)
    n, dx = 64, 1e-4
    c = (1500 + 80 * rng.standard_normal((n, n))).astype(np.float32)
    g = KWaveGrid(n, dx, n, dx)
    g.makeTime(float(c.max()), cfl=0.3)
    g.setTime(90, g.dt)
    pts = rng.uniform(-20 * dx, 20 * dx, size=(2, 40)).astype(np.float32)
    p0 = makeDisc(n, n, 24, 38, 3) * 1e3
    b = DescBuilder(g, KWaveMedium(c, 1000.0), KWaveSource(p0=p0), KWaveSensor(mask=pts, record=RecordField.p),
                    SimulationOptions(pmlSize=6, smoothP0=False))
    ref, _ = oracle.run(b)
    out = run_gpu(b)
    assert out["p"].shape == (40, 90)
    _rowwise_order_check(out["p"], ref["p"])
