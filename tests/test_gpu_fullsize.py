"""Configuration 2 at its full size: SME level 4 on the 1400x1400 jittered
grid (3,914,402 cells), the bench's workload.

* the configuration's 100 steps against the oracle on the same mesh, every
  step bit for bit (the oracle takes a few seconds per step at this size);
* the same 100 steps free running, through size-independent properties: mass
  conserved to rounding with reflective walls, depths non-negative and
  finite, the bathymetry untouched, the health counters clean;
* the lake at rest stays at rest at first order to 1e-14;
* both positivity variants keep depths non-negative and conserve mass.
"""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models
from zoomy_dmplex_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    return cases.roofline_l4(1400)


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def test_hundred_steps_per_step_against_oracle(case):
    """All 100 steps of the configuration, every step compared with the
    oracle on the same mesh: the oracle runs free, the GPU takes the oracle's
    dt each step, and the states must agree bit for bit (no FMA contraction,
    IEEE division and square root on both sides; the level-4 plugins call no
    cbrt).  The oracle needs a few seconds per step on the host's cores."""
    p = _params(case)
    O.set_threads(0)
    o = O.Oracle(case.model, case.mesh.as_abi_arrays(), case.settings.to_struct(), p)
    o.set_state(case.q0)
    g = Solver(case.model, case.mesh, case.settings, p)
    g.set_state(case.q0)
    assert g.time()[1] == pytest.approx(o.time()[1], rel=1e-12)
    for k in range(case.steps):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        qg, qo = g.get_state(), o.get_state()
        if not np.array_equal(qg, qo):
            e = np.abs(qg - qo).max(axis=0) / np.maximum(np.abs(qo).max(axis=0), 1e-300)
            raise AssertionError("step %d: per-variable relative max error %s" % (k + 1, e))
        assert g.time()[0] == o.time()[0]
    assert case.steps == 100
    assert g.time()[1] == pytest.approx(o.time()[1], rel=1e-12)
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0
    g.close()


def test_hundred_steps_conserve_mass(case):
    g = Solver(case.model, case.mesh, case.settings, _params(case))
    g.set_state(case.q0)
    vol = case.mesh.cell_volume
    m0 = np.sum(g.get_state()[:, 1] * vol)
    g.step(100)
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0 and d.n_newton_unconverged == 0
    q = g.get_state()
    assert np.all(np.isfinite(q)) and q[:, 1].min() >= 0.0
    assert np.array_equal(q[:, 0], case.q0[:, 0])                     # b is not evolved
    assert abs(np.sum(q[:, 1] * vol) - m0) <= 1e-12 * m0
    g.close()


def test_lake_at_rest_first_order(case):
    q = case.q0.copy()
    q[:, 1] = 1.0 - q[:, 0]
    q[:, 2:] = 0.0
    st = dataclasses.replace(case.settings, reconstruction_order=1)
    g = Solver(case.model, case.mesh, st, _params(case))
    g.set_state(q)
    g.step(5)
    r = g.get_state()
    assert np.abs(r[:, 0] + r[:, 1] - 1.0).max() < 1e-14
    assert np.abs(r[:, 2:]).max() < 1e-14
    g.close()


@pytest.mark.parametrize("pos", ["zhang_shu", "mood"])
def test_positivity_variants_at_full_size(case, pos):
    """The positivity variants on the same mesh: 20 steps with depths
    non-negative, mass conserved to rounding and the counters clean."""
    st = dataclasses.replace(case.settings, positivity=pos)
    g = Solver(case.model, case.mesh, st, _params(case))
    g.set_state(case.q0)
    vol = case.mesh.cell_volume
    m0 = np.sum(g.get_state()[:, 1] * vol)
    g.step(20)
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0
    q = g.get_state()
    assert q[:, 1].min() >= 0.0
    assert abs(np.sum(q[:, 1] * vol) - m0) <= 1e-12 * m0
    g.close()
