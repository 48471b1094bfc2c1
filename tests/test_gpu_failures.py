"""Failure paths of the C ABI on the GPU, made without a GPU fault.

The reference's only error path is `precondition` / `fatalError` (KSpaceFirstOrder.swift:105,
358-359), which traps; the library returns status codes instead. These tests reach the codes
beyond KW_ERR_INVALID:
  KW_ERR_TIMEOUT    the TMA-fed column pass withholds each CTA's first tile copy and its consumers
                    wait at most ~20 us for it (KW_TEST_STALL_COLUMN_PASS): nothing completes that
                    barrier, so the bounded wait runs out; the kernel records the code, its producer
                    drains the copies it did issue and returns, and the context stays usable;
  KW_ERR_NONFINITE  an unstable run (1 GPa initial pressure with B/A = 10 at CFL 1.5: the nonlinear
                    factor blows the update up within a few steps) stops at the run's next
                    non-finite poll instead of running on;
  KW_ERR_OOM        a simulated device-allocation failure (KW_TEST_FAIL_ALLOC), which the engine
                    reports and cleans up after.
"""
import numpy as np
import pytest

import oracle
from cases import rel_l2
from kwave import (DescBuilder, KWaveError, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, RecordField,
                   SimulationOptions, abi, makeBall, makeCircle, makeDisc)
from kwave.runtime import Context

pytestmark = pytest.mark.gpu


def _run(builder):
    sim = Context.default().create_sim(builder)
    try:
        sim.run()
        return sim.output("pFinal"), sim.t
    finally:
        sim.close()


def _tma_case():
    # 3D with B = 32: the in-place column passes along B run the TMA-fed kernel
    shape = (20, 32, 24)
    g = KWaveGrid(shape[0], 1e-4, shape[1], 1e-4, shape[2], 1e-4)
    g.setTime(3, 2e-8)
    return DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeBall(*shape, radius=3) * 1.0),
                       KWaveSensor(), SimulationOptions(pmlSize=4, smoothP0=False))


def test_bounded_wait_timeout_returns_status(monkeypatch):
    b = _tma_case()
    monkeypatch.setenv("KW_TEST_STALL_COLUMN_PASS", "1")
    with pytest.raises(KWaveError) as e:
        _run(b)
    assert e.value.status == abi.KW_ERR_TIMEOUT, e.value
    # the context is still usable: the same run with the default limit matches the oracle
    monkeypatch.delenv("KW_TEST_STALL_COLUMN_PASS")
    pf, _ = _run(b)
    ref, _ = oracle.run(b)
    assert rel_l2(pf, ref["pFinal"]) < 1e-4


def test_unstable_run_returns_nonfinite():
    n = 64
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.setTime(300, 1.5 * 1e-4 / 1500.0)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0, bOnA=10.0), KWaveSource(p0=makeDisc(n, n, radius=4) * 1e9),
                    KWaveSensor(mask=makeCircle(n, n, radius=20), record=RecordField.p),
                    SimulationOptions(pmlSize=8, smoothP0=False))
    sim = Context.default().create_sim(b)
    try:
        with pytest.raises(KWaveError) as e:
            sim.run()
        assert e.value.status == abi.KW_ERR_NONFINITE, e.value
        # stopped at a poll (every 64 steps), well before the end of the run
        assert 0 < sim.t < 300, sim.t
        assert sim.t % 64 == 0, sim.t
    finally:
        sim.close()


@pytest.mark.parametrize("nth", [1, 5, 12])
def test_allocation_failure_returns_oom(monkeypatch, nth):
    n = 32
    g = KWaveGrid(n, 1e-4, n, 1e-4)
    g.setTime(10, 2e-8)
    b = DescBuilder(g, KWaveMedium(1500.0, 1000.0), KWaveSource(p0=makeDisc(n, n, radius=3)), KWaveSensor())
    monkeypatch.setenv("KW_TEST_FAIL_ALLOC", str(nth))
    with pytest.raises(KWaveError) as e:
        Context.default().create_sim(b)
    assert e.value.status == abi.KW_ERR_OOM, e.value
    monkeypatch.delenv("KW_TEST_FAIL_ALLOC")
    pf, t = _run(b)
    assert t == 10 and np.isfinite(pf).all()
