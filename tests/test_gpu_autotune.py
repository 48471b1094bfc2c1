"""The autotuner of the operator column pass (kw_tune.cpp) and the variants it chooses among.

Every variant (values per thread R1, CTAs per SM) of the lengths the benchmarks run is forced in
turn: variants with the default's R1 must reproduce the default run bit for bit (same arithmetic,
other launch shape); the others split the transform into other radix stages and must agree to
1e-5 relative L2 (the FP32 rounding of another split; all agree with the FP64 oracle at 1e-4).
With tuning on, the chosen variants are written to the JSON cache and the run still matches the
oracle.
"""
import json

import numpy as np
import pytest

import oracle
from cases import rel_l2
from kwave.runtime import Context
from test_gpu_parity import _reg_case, compare

pytestmark = pytest.mark.gpu

# (shape, operator-axis length): 3D passes run along A, 2D along B
SHAPES = [((256, 24, 32), 256), ((128, 24, 32), 128), ((192, 16, 24), 192), ((512, 64), 512)]
# (r1, minb); minb -1 is the TMA-fed warp-specialised kernel (3D passes along A of 128 and 256),
# minb -10 - m the persistent kernel with m CTAs per SM that prefetches its next tile into L2
VARIANTS = {16: [], 256: [(16, 3), (16, 2), (8, 3), (8, 4), (16, -13), (16, -12), (8, -13), (16, -1)],
            128: [(16, 3), (16, 2), (8, 3), (8, 4), (16, -13), (16, -1)],
            192: [(12, 3), (12, 2), (12, 4), (12, -13)],
            512: [(16, 0), (16, 2), (8, 2), (8, 3), (8, 4), (16, -12), (8, -13)]}


def _run(b):
    sim = Context.default().create_sim(b)
    try:
        sim.run()
        return sim.output("p"), sim.output("pFinal")
    finally:
        sim.close()


@pytest.mark.parametrize("shape,n", SHAPES)
def test_every_variant_matches_the_default(shape, n, monkeypatch):
    monkeypatch.setenv("KW_AUTOTUNE", "0")
    b = _reg_case(shape, sum(shape) + 3, 6)
    p_ref, pf_ref = _run(b)
    default_r1 = VARIANTS[n][0][0]
    for r1, minb in VARIANTS[n]:
        monkeypatch.setenv("KW_COLOP_VARIANT", f"{r1},{minb}")
        p, pf = _run(b)
        if r1 == default_r1:
            assert np.array_equal(p, p_ref) and np.array_equal(pf, pf_ref), (r1, minb)
        else:
            assert rel_l2(p, p_ref) < 1e-5 and rel_l2(pf, pf_ref) < 1e-5, (r1, minb, rel_l2(p, p_ref))
    monkeypatch.delenv("KW_COLOP_VARIANT")


def test_tuned_choices_are_cached_and_match_the_oracle(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("KW_TUNE_CACHE", str(cache))
    monkeypatch.setenv("KW_AUTOTUNE", "1")
    b = _reg_case((256, 24, 32), 11, 6)
    sim = Context.default().create_sim(b)
    try:
        sim.run()
        out = {k: v for k, v in vars(sim.outputs()).items()}
    finally:
        sim.close()
    ref, _ = oracle.run(b)
    compare(out, ref)
    doc = json.loads(cache.read_text())
    keys = [k for k in doc["choices"] if k.startswith("colop/256/0/")]
    assert keys, doc
    for k in keys:
        c = doc["choices"][k]
        assert (c["r1"], c["minb"]) in VARIANTS[256] and c["us"] > 0
