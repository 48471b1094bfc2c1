"""Scheduling choices that must not change a single bit of the results.

The tile maps' traversal order (KW_MAP_ORDER: alternating by default, 0 forwards, 2 column-chunk
major), the C2R epilogues' L2 prefetch (KW_C2R_PREFETCH=0 off), the row kernels' prefetch of the
next wave's rows (KW_ROW_AHEAD=0 off) and programmatic dependent launch
(KW_PDL=1 on) only change when and where the same CTAs run, never what they compute: every tile is
independent and every kernel still runs after the whole of the previous one. A 3D power-law + B/A
case with an additive source on register kernels only (64 x 48 x 64), one with staged column
kernels and a partial last row tile (40 x 36 x 64), and a 2D case must give bit-identical p series
and pFinal under each setting.
"""
import numpy as np
import pytest

from kwave.runtime import Context
from test_gpu_parity import _reg_case

pytestmark = pytest.mark.gpu

CASES = [((64, 48, 64), 6), ((40, 36, 64), 5), ((100, 128), 6)]
SETTINGS = [("KW_MAP_ORDER", "0"), ("KW_MAP_ORDER", "2"), ("KW_C2R_PREFETCH", "0"), ("KW_ROW_AHEAD", "0"), ("KW_PDL", "1")]


def _run(b):
    sim = Context.default().create_sim(b)
    try:
        sim.run()
        return sim.output("p"), sim.output("pFinal")
    finally:
        sim.close()


@pytest.mark.parametrize("shape,pml", CASES, ids=lambda v: str(v))
def test_results_do_not_depend_on_scheduling(shape, pml, monkeypatch):
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    b = _reg_case(shape, sum(shape), pml)
    p_ref, pf_ref = _run(b)
    for name, value in SETTINGS:
        monkeypatch.setenv(name, value)
        p, pf = _run(b)
        monkeypatch.delenv(name)
        assert np.array_equal(p, p_ref) and np.array_equal(pf, pf_ref), (name, value)
