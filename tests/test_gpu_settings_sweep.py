"""GPU step against the oracle across the solver settings the reference's
JSON offers: SSP stage counts 2, 3 and 5 (5 is the reference default), the
limiter on or off, Green-Gauss or least-squares gradients, order 1 or 2, and
the positivity variants -- bit for bit on a small level-2 case (its plugins
call no cbrt), ten steps with the oracle's dts."""
import itertools

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases
from zoomy_dmplex_b200.solver import Solver

from test_gpu_parity import params

pytestmark = pytest.mark.gpu

CASE = cases.level2(24)
COMBOS = [c for c in itertools.product((2, 3, 5), ("tvd", "none"), ("green_gauss", "least_squares"), (1, 2),
                                       ("none", "mood"))
          if not (c[3] == 1 and (c[0] != 2 or c[1] != "tvd" or c[2] != "green_gauss"))]


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


@pytest.mark.parametrize("stages,limiter,gradient,order,positivity", COMBOS)
def test_settings_bitwise(stages, limiter, gradient, order, positivity):
    s = cases.default_settings(ssp_stages=stages, limiter=limiter, gradient=gradient, reconstruction_order=order,
                               positivity=positivity)
    p = params(CASE.model, CASE.params)
    g = Solver(CASE.model, CASE.mesh, s, p)
    o = O.Oracle(CASE.model, CASE.mesh.as_abi_arrays(), s.to_struct(), p)
    g.set_state(CASE.q0)
    o.set_state(CASE.q0)
    assert g.time()[1] == o.time()[1]
    for k in range(10):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        assert np.array_equal(g.get_state(), o.get_state()), "step %d" % k
