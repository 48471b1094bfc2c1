"""Device discrete adjoint (kw_adjoint_run through the C ABI) against the FP64 oracle adjoint and
FP64 central finite differences of the oracle's misfit.

Tolerances (FP32 device arithmetic): misfit relative error <= 1e-3; gradient fields (c0, p0, rho0)
relative L2 <= 2e-3 against the FP64 adjoint; directional derivatives within 1e-3 of the finite differences
(2e-3 for the replica of the 512^2 configuration, whose 1 % speed error leaves a small misfit);
the checkpoint policies agree to 1e-5.
"""
import numpy as np
import pytest

import oracle
from adjoint_cases import builder, fd_misfit_diff, problem
from cases import rel_l2
from kwave import KWaveError, abi
from kwave.runtime import Context

pytestmark = pytest.mark.gpu

CASES = [
    ((48, 40), dict(absorb="powerlaw", nonlinear=False, cartesian=True, nt=60)),
    ((40, 36), dict(absorb="none", nonlinear=True, cartesian=False, nt=50)),
    ((40, 36), dict(absorb="stokes", nonlinear=False, cartesian=True, nt=50)),
    ((36, 32), dict(absorb="nodispersion", nonlinear=True, cartesian=False, nt=40, no_p0=True)),
    ((96,), dict(absorb="powerlaw", nonlinear=True, cartesian=False, nt=60)),
    ((20, 18, 16), dict(absorb="powerlaw", nonlinear=True, cartesian=True, nt=30)),
]


def gpu_adjoint(shape, c, p0, data, kw, grad_rho0=False, **opt):
    return Context.default().adjoint(builder(shape, c, p0, **kw), data, grad_c0=True, grad_p0=p0 is not None,
                                     grad_rho0=grad_rho0, **opt)


@pytest.mark.parametrize("shape,kw", CASES)
def test_device_adjoint_matches_fp64_adjoint_and_differences(shape, kw):
    c, p0, data, kw = problem(shape, **kw)
    L, gc, gp = oracle.adjoint(builder(shape, c, p0, **kw), data)
    r = gpu_adjoint(shape, c, p0, data, kw)
    assert abs(r["misfit"] - L) <= 1e-3 * L, (r["misfit"], L)
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)
    if p0 is not None:
        assert rel_l2(r["grad_p0"], gp) < 2e-3, rel_l2(r["grad_p0"], gp)
    rng = np.random.default_rng(3)
    for _ in range(2):
        dL, dx = fd_misfit_diff(shape, c, p0, data, rng.standard_normal(shape), 0.1, "c", kw)
        assert abs(dL - np.sum(r["grad_c0"] * dx)) <= 1e-3 * abs(dL)


@pytest.mark.parametrize("shape,kw", [((40, 64), dict(absorb="powerlaw", nonlinear=True, cartesian=True, nt=50)),
                                      CASES[3], CASES[4], ((16, 20, 32), dict(absorb="powerlaw", nonlinear=False, nt=30))])
def test_fused_reverse_eos_matches_fp64_adjoint(shape, kw, monkeypatch):
    # the absorption job's C2R epilogue carries the reverse equation of state (chosen by default
    # on large grids only; forced here)
    monkeypatch.setenv("KW_ADJOINT_FUSED_EOS", "1")
    c, p0, data, kw = problem(shape, **kw)
    L, gc, gp = oracle.adjoint(builder(shape, c, p0, **kw), data)
    r = gpu_adjoint(shape, c, p0, data, kw)
    assert abs(r["misfit"] - L) <= 1e-3 * L
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)
    if p0 is not None:
        assert rel_l2(r["grad_p0"], gp) < 2e-3, rel_l2(r["grad_p0"], gp)


@pytest.mark.parametrize("cola", ["0", "1"])
@pytest.mark.parametrize("shape,kw", [((48, 64), dict(absorb="powerlaw", nonlinear=True, nt=40)),
                                      ((16, 20, 32), dict(absorb="stokes", nonlinear=True, nt=30))])
def test_fan_in_sum_matches_per_component_sum(shape, kw, cola, monkeypatch):
    # lambda_p = sum_a D-_a w_a: one inverse of the summed spectra against one inverse per component
    # (operator pass on the one-tile-per-CTA or the double-buffered column kernel)
    monkeypatch.setenv("KW_COLA", cola)
    c, p0, data, kw = problem(shape, **kw)
    monkeypatch.setenv("KW_ADJOINT_FANIN", "1")
    r1 = gpu_adjoint(shape, c, p0, data, kw)
    monkeypatch.setenv("KW_ADJOINT_FANIN", "0")
    r0 = gpu_adjoint(shape, c, p0, data, kw)
    assert rel_l2(r1["grad_c0"], r0["grad_c0"]) < 1e-4, rel_l2(r1["grad_c0"], r0["grad_c0"])
    if p0 is not None:
        assert rel_l2(r1["grad_p0"], r0["grad_p0"]) < 1e-4


@pytest.mark.parametrize("shape,kw", [((40, 36), dict(absorb="powerlaw", nonlinear=True, nt=45)),
                                      ((16, 20, 32), dict(absorb="stokes", nonlinear=True, nt=30))])
def test_overlapped_reverse_sweep_matches_sequential(shape, kw, monkeypatch):
    # segment c + 1 reversed on a second stream while segment c is recomputed (one tape bank whose
    # slots alternate direction) gives the same gradient as running them one after the other
    c, p0, data, kw = problem(shape, **kw)
    monkeypatch.setenv("KW_ADJOINT_OVERLAP", "1")
    r1 = gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_INTERVAL, interval=6)
    monkeypatch.setenv("KW_ADJOINT_OVERLAP", "0")
    r0 = gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_INTERVAL, interval=6)
    assert r1["checkpoints"] == r0["checkpoints"] > 2
    assert rel_l2(r1["grad_c0"], r0["grad_c0"]) < 1e-6
    assert rel_l2(r1["grad_p0"], r0["grad_p0"]) < 1e-6
    assert r1["misfit"] == r0["misfit"]


def test_checkpoint_policies_agree():
    shape = (40, 36)
    c, p0, data, kw = problem(shape, absorb="powerlaw", nonlinear=True, nt=45)
    runs = [gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_SQRT),
            gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_INTERVAL, interval=8),
            gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_STORE_ALL),
            gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_BUDGET, memory_budget=1e6)]
    assert runs[0]["interval"] == 7 and runs[0]["checkpoints"] == 7
    assert runs[2]["checkpoints"] == 0
    for r in runs[1:]:
        assert rel_l2(r["grad_c0"], runs[0]["grad_c0"]) < 1e-5
        assert rel_l2(r["grad_p0"], runs[0]["grad_p0"]) < 1e-5
        assert abs(r["misfit"] - runs[0]["misfit"]) <= 1e-6 * runs[0]["misfit"]


def test_adjoint_rejects_unsupported():
    shape = (32, 32)
    c, p0, data, kw = problem(shape, absorb="none")
    b = builder(shape, c, p0, **kw)
    b.desc.p_mode = 0   # Dirichlet pressure source
    with pytest.raises(KWaveError) as e:
        Context.default().adjoint(b, data)
    assert e.value.status == abi.KW_ERR_UNSUPPORTED
    b = builder(shape, c, p0, **kw)
    b.desc.axisymmetric = 1
    with pytest.raises(KWaveError) as e:
        Context.default().adjoint(b, data)
    assert e.value.status == abi.KW_ERR_UNSUPPORTED


def test_adjoint2d_configuration_replica():
    """The 512^2 adjoint configuration at 128^2 and 200 steps (same construction, scaled): the
    device gradient against the FP64 adjoint and against FP64 central differences along smoothed
    random directions of unit norm with step 1e-4 max|c0|."""
    from kwave import workloads
    from kwave.workloads import _gauss_smooth_wrap
    bp, bt = workloads.adjoint2d(128, 200)
    data = oracle.run(bt)[0]["p"]
    c = np.asarray(bp.medium.soundSpeed, np.float64)
    L, gc, gp = oracle.adjoint(bp, data)
    r = Context.default().adjoint(bp, data, grad_c0=True, grad_p0=True)
    assert abs(r["misfit"] - L) <= 1e-3 * L
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)
    assert rel_l2(r["grad_p0"], gp) < 2e-3, rel_l2(r["grad_p0"], gp)
    rng = np.random.default_rng(17)
    eps = 1e-4 * np.abs(c).max()
    for _ in range(4):
        v = _gauss_smooth_wrap(rng.standard_normal(c.shape), 4.0)
        v /= np.linalg.norm(v)
        xp = (c + eps * v).astype(np.float32)
        xm = (c - eps * v).astype(np.float32)
        lp = oracle.adjoint(_with_c(bp, xp), data)[0]
        lm = oracle.adjoint(_with_c(bp, xm), data)[0]
        dL = lp - lm
        # the misfit of a 1 % speed error is small next to the signal, so FP32 rounding of the
        # recorded pressure reaches ~1e-3 of the residual: 2e-3 here
        assert abs(dL - np.sum(r["grad_c0"] * (xp.astype(np.float64) - xm))) <= 2e-3 * abs(dL)


def _with_c(b, c):
    from kwave import DescBuilder, KWaveMedium
    m = b.medium
    return DescBuilder(b.grid, KWaveMedium(c, m.density, alphaCoeff=m.alphaCoeff, alphaPower=m.alphaPower,
                                           alphaMode=m.alphaMode, bOnA=m.bOnA), b.source, b.sensor, b.options)


def test_adjoint3d_configuration_replica():
    """The 384^3 forward + adjoint configuration at 48^3 and 40 steps (same construction, scaled:
    layers, spheres, focused element array, receive plane): the device gradient against the FP64
    adjoint, with the memory-budget checkpoint schedule."""
    from kwave import workloads
    bp, bt = workloads.adjoint3d(48, 40)
    data = oracle.run(bt)[0]["p"]
    L, gc, _ = oracle.adjoint(bp, data)
    r = Context.default().adjoint(bp, data, grad_c0=True, policy=abi.KW_CHECKPOINT_BUDGET, memory_budget=5e7)
    assert r["checkpoints"] > 0
    assert abs(r["misfit"] - L) <= 1e-3 * L
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)


@pytest.mark.parametrize("shape,kw,fused_eos", [
    (CASES[0][0], CASES[0][1], "0"), (CASES[1][0], CASES[1][1], "0"), (CASES[2][0], CASES[2][1], "0"),
    (CASES[3][0], CASES[3][1], "0"), (CASES[4][0], CASES[4][1], "0"), (CASES[5][0], CASES[5][1], "0"),
    ((40, 64), dict(absorb="powerlaw", nonlinear=True, cartesian=True, nt=50), "1"),
    ((16, 20, 32), dict(absorb="powerlaw", nonlinear=False, nt=30), "1")])
def test_device_density_gradient(shape, kw, fused_eos, monkeypatch):
    # dL/drho0 (dt rho0 nl, dt / staggerDensity(rho0), rho0 div, B/A S^2 / (2 rho0)) against the FP64
    # adjoint at 2e-3 relative L2 and FP64 central differences at 2e-3 (the density directional
    # derivatives cancel more than the sound speed's, so the FP32 rounding of the device gradient
    # shows at the 1e-3 level there); rows of 64 points take the register
    # kernels with the reverse equation of state fused (forced here), the others the elementwise ones
    monkeypatch.setenv("KW_ADJOINT_FUSED_EOS", fused_eos)
    c, p0, data, kw = problem(shape, **kw)
    L, gc, gp, gr = oracle.adjoint(builder(shape, c, p0, **kw), data, grad_rho0=True)
    r = gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True)
    assert abs(r["misfit"] - L) <= 1e-3 * L
    assert rel_l2(r["grad_c0"], gc) < 2e-3, rel_l2(r["grad_c0"], gc)
    e_l2 = rel_l2(r["grad_rho0"], gr)
    assert e_l2 < 2e-3, e_l2
    rng = np.random.default_rng(4)
    for _ in range(2):
        v = rng.standard_normal(shape)
        dL, dx = fd_misfit_diff(shape, c, p0, data, v, 0.1, "rho", kw)
        e_fd = abs(dL - np.sum(r["grad_rho0"] * dx)) / abs(dL)
        e_64 = abs(np.sum((r["grad_rho0"] - gr) * v)) / abs(np.sum(gr * v))   # against the FP64 adjoint
        print(f"\n{shape} {kw}: rel L2 {e_l2:.2e}, directional vs FD {e_fd:.2e}, vs FP64 adjoint {e_64:.2e}")
        assert e_fd <= 2e-3, (e_fd, e_64)


def test_density_gradient_checkpoint_policies_agree():
    # p(t-1) of a segment's first step comes from its checkpoint, of the others from the tape;
    # the overlapped and sequential reverse sweeps agree too
    shape = (40, 36)
    c, p0, data, kw = problem(shape, absorb="powerlaw", nonlinear=True, nt=45)
    runs = [gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True, policy=abi.KW_CHECKPOINT_STORE_ALL),
            gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True, policy=abi.KW_CHECKPOINT_SQRT),
            gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True, policy=abi.KW_CHECKPOINT_INTERVAL, interval=6)]
    for r in runs[1:]:
        assert r["checkpoints"] > 2
        assert rel_l2(r["grad_rho0"], runs[0]["grad_rho0"]) < 1e-5
        assert rel_l2(r["grad_c0"], runs[0]["grad_c0"]) < 1e-5


@pytest.mark.parametrize("snapshots", [1, 3, 6])
def test_revolve_matches_store_all(snapshots):
    # the binomial (revolve) schedule with 1, 3 and 6 state snapshots (one tape slot) against
    # keeping every state: the 48^3 power-law + B/A problem, gradients of c0, p0 and rho0
    shape = (48, 48, 48)
    c, p0, data, kw = problem(shape, absorb="powerlaw", nonlinear=True, cartesian=True, nt=40)
    ref = gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True, policy=abi.KW_CHECKPOINT_STORE_ALL)
    r = gpu_adjoint(shape, c, p0, data, kw, grad_rho0=True, policy=abi.KW_CHECKPOINT_REVOLVE, interval=snapshots)
    assert r["checkpoints"] == snapshots and r["interval"] == 0
    assert abs(r["misfit"] - ref["misfit"]) <= 1e-6 * ref["misfit"]
    for g in ("grad_c0", "grad_p0", "grad_rho0"):
        assert rel_l2(r[g], ref[g]) < 1e-5, (g, rel_l2(r[g], ref[g]))


def test_budget_falls_back_to_revolve():
    # a memory budget below every uniform interval's needs (checkpoints + tape slots) but above a
    # few snapshots takes the binomial schedule
    shape = (40, 36)
    c, p0, data, kw = problem(shape, absorb="powerlaw", nonlinear=True, nt=45)
    fb = 40 * 36 * 4
    ref = gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_STORE_ALL)
    r = gpu_adjoint(shape, c, p0, data, kw, policy=abi.KW_CHECKPOINT_BUDGET, memory_budget=60.0 * fb)
    assert r["interval"] == 0 and r["checkpoints"] == 7   # (60 - 5 tape - 2) // 7 fields per snapshot
    assert rel_l2(r["grad_c0"], ref["grad_c0"]) < 1e-5
    assert rel_l2(r["grad_p0"], ref["grad_p0"]) < 1e-5
