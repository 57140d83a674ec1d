"""RefreshDerivativeAux on the GPU (derivative_aux_kernel) against the
oracle's restatement: the 1-D level-0 model's derivative aux slots after
set_state, after steps on the CUDA graph and after zsme_update_state are
bit-identical to the oracle's; the state does not depend on the refresh;
2-D models, which have no derivative slots, launch nothing extra."""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, mesh as meshmod, models
from zoomy_dmplex_b200.solver import Solver

from test_derivative_aux import _setup

pytestmark = pytest.mark.gpu


def _pair(m, q, p, refresh=True, **kw):
    st = dataclasses.replace(cases.default_settings(**kw), refresh_derivative_aux=refresh)
    g = Solver("sme1d_l0_malpasset", m, st, p)
    o = O.Oracle("sme1d_l0_malpasset", m.as_abi_arrays(), st.to_struct(), p)
    g.set_state(q)
    o.set_state(q)
    return g, o


@pytest.mark.parametrize("order", [1, 2])
def test_gpu_derivative_aux_matches_oracle(order):
    m, q, p = _setup()
    g, o = _pair(m, q, p, reconstruction_order=order)
    assert np.array_equal(g.get_aux(), o.get_aux())
    for k in range(3):
        g.step(5)
        o.step(5)
        assert np.array_equal(g.get_state(), o.get_state()), k
        assert np.array_equal(g.get_aux(), o.get_aux()), k
    assert np.abs(g.get_aux()[:, :3]).max() > 0.0
    g.update_state()
    o.update_state()
    assert np.array_equal(g.get_aux(), o.get_aux())


def test_gpu_state_independent_of_refresh():
    m, q, p = _setup()
    on, _ = _pair(m, q, p, True)
    off, _ = _pair(m, q, p, False)
    on.step(20)
    off.step(20)
    assert np.array_equal(on.get_state(), off.get_state())
    assert np.all(off.get_aux()[:, :3] == 0.0)
    assert on.launches_per_step() == off.launches_per_step() + 4   # two stages, before and after finalize


def test_gpu_no_derivative_slots_in_2d_models():
    c = cases.level2(24)
    names, vals = models.parameter_table(c.model)
    p = np.array(vals, float)
    on = Solver(c.model, c.mesh, dataclasses.replace(c.settings, refresh_derivative_aux=True), p)
    off = Solver(c.model, c.mesh, dataclasses.replace(c.settings, refresh_derivative_aux=False), p)
    assert on.launches_per_step() == off.launches_per_step()
