"""The FP64 discrete adjoint of the oracle against FP64 central finite differences of the oracle's
own misfit (the check that pins the adjoint equations before the device adjoint is compared
with them).

Tolerance: relative error of the directional derivative <= 2e-6 against central differences
extrapolated (Richardson) from steps 0.2 and 0.1 m/s (sound speed), 2 and 1 x 1e3 Pa (initial
pressure), 0.2 and 0.1 kg/m^3 (density).
"""
import numpy as np
import pytest

import oracle
from adjoint_cases import fd_misfit_diff, problem, builder

CASES = [
    ((32, 28), dict(absorb="none", nonlinear=False, cartesian=True)),
    ((32, 28), dict(absorb="powerlaw", nonlinear=True, cartesian=True)),
    ((30, 26), dict(absorb="stokes", nonlinear=True, cartesian=False)),
    ((30, 26), dict(absorb="nodispersion", nonlinear=False, cartesian=False, no_p0=True)),
    ((64,), dict(absorb="powerlaw", nonlinear=True, cartesian=False)),
    ((14, 12, 12), dict(absorb="powerlaw", nonlinear=False, cartesian=True, nt=24)),
]


def richardson_error(shape, c, p0, data, g, v, eps, which, kw):
    """Relative error of <g, dx> against central differences at eps and eps/2, combined so that
    the O(eps^2) truncation cancels."""
    r = []
    for e in (eps, eps / 2):
        dL, dx = fd_misfit_diff(shape, c, p0, data, v, e, which, kw)
        r.append((dL - np.sum(g * dx)) / dL)
    return abs((4 * r[1] - r[0]) / 3)


@pytest.mark.parametrize("shape,kw", CASES)
def test_oracle_adjoint_matches_central_differences(shape, kw):
    rng = np.random.default_rng(11)
    c, p0, data, kw = problem(shape, **kw)
    L, gc, gp, gr = oracle.adjoint(builder(shape, c, p0, **kw), data, grad_rho0=True)
    assert L > 0
    assert richardson_error(shape, c, p0, data, gc, rng.standard_normal(shape), 0.2, "c", kw) < 2e-6
    if p0 is not None:
        assert richardson_error(shape, c, p0, data, gp, rng.standard_normal(shape) * 1e3, 2.0, "p", kw) < 2e-6
    # density: steps 0.2 and 0.1 kg/m^3
    assert richardson_error(shape, c, p0, data, gr, rng.standard_normal(shape), 0.2, "rho", kw) < 2e-6


def test_oracle_adjoint_rejects_unsupported_sources():
    shape = (24, 24)
    c, p0, data, kw = problem(shape, absorb="none")
    b = builder(shape, c, p0, **kw)
    b.desc.p_mode = 0   # Dirichlet
    with pytest.raises(oracle.OracleError):
        oracle.adjoint(b, data)
