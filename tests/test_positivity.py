"""The positivity variants of the order-2 step (settings.solver.positivity),
on the oracle.

* zhang_shu: the eta-well-balanced reconstruction with the Zhang-Shu theta,
  CFL clamped to 1/6 at order 2 (MUSCLSolver.hpp:33-38);
* mood: the same reconstruction without theta at full CFL, and every cell
  whose depth ends below -1e-10 replaced by its first-order forward-Euler
  update from the step's start state (MUSCLSolver.hpp:150-170, 197-229).

The MOOD test rebuilds the step from the oracle's own right-hand sides, the
order-2 candidate from the configured rhs and the override from an order-1
rhs, so the per-cell override path is checked against the whole-mesh
first-order path.
"""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


def params(case):
    names, vals = models.parameter_table(case.model)
    for k, v in case.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def oracle(case, **kw):
    st = dataclasses.replace(case.settings, **kw).to_struct()
    o = O.Oracle(case.model, case.mesh.as_abi_arrays(), st, params(case))
    o.set_state(case.q0)
    return o


def test_zhang_shu_clamps_cfl_at_order_two():
    c = cases.wet_dry_patchwork(16)
    dt_none = oracle(c, cfl=0.45).time()[1]
    dt_zs = oracle(c, cfl=0.45, positivity="zhang_shu").time()[1]
    assert dt_zs == pytest.approx(dt_none * (1.0 / 6.0) / 0.45, rel=1e-13)
    # below 1/6, and at order 1, the configured CFL stands
    assert oracle(c, cfl=0.1, positivity="zhang_shu").time()[1] == pytest.approx(
        oracle(c, cfl=0.1).time()[1], rel=1e-15)
    o1 = oracle(c, cfl=0.45, positivity="zhang_shu", reconstruction_order=1)
    assert o1.time()[1] == oracle(c, cfl=0.45, reconstruction_order=1).time()[1]


def test_variants_keep_depth_nonnegative():
    """At CFL 1.5 the limited order-2 step drives depths negative; Zhang-Shu
    (at its clamped CFL) and MOOD keep every depth >= 0, MOOD by overriding
    cells."""
    c = cases.wet_dry_patchwork(24)
    hmin = {}
    for pos in ("none", "zhang_shu", "mood"):
        o = oracle(c, positivity=pos)
        lo = np.inf
        for _ in range(c.steps):
            o.step(1)
            s = o.get_state()
            assert np.all(np.isfinite(s))
            lo = min(lo, s[:, 1].min())
        hmin[pos] = lo
        if pos == "mood":
            assert o.mood_cells() > 0
        else:
            assert o.mood_cells() == 0
    assert hmin["none"] < -1e-4
    assert hmin["zhang_shu"] >= 0.0 and hmin["mood"] >= 0.0


def test_mood_step_is_candidate_or_first_order_update():
    c = cases.wet_dry_patchwork(24)
    st = dataclasses.replace(c.settings, positivity="mood").to_struct()
    st.source = 0
    p = params(c)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st, p)
    o.set_state(c.q0)
    x0 = o.get_state()                      # constrained start state
    t0, dt = o.time()
    o.step(1)
    x1 = o.get_state()
    # order-2 candidate: SSP-RK(2,2) over the configured rhs (well-balanced, no theta)
    f0 = o.rhs(x0, t0)
    w1 = x0 + dt / 1.0 * f0
    f1 = o.rhs(w1, t0 + dt)
    cand = 0.5 * w1 + (dt / 2.0) * f1 + 0.5 * x0
    bad = cand[:, 1] < -1.0e-10
    assert bad.sum() == o.mood_cells() > 0
    # first-order update from the start state (piecewise constant)
    s1 = dataclasses.replace(c.settings, positivity="mood", reconstruction_order=1).to_struct()
    s1.source = 0
    o1 = O.Oracle(c.model, c.mesh.as_abi_arrays(), s1, p)
    euler = x0 + dt * o1.rhs(x0, t0)
    expect = np.where(bad[:, None], euler, cand)
    ref = O.Oracle(c.model, c.mesh.as_abi_arrays(), s1, p)
    ref.set_state(expect)                   # the constraints, as after the override
    assert np.array_equal(x1, ref.get_state())
    assert x1[:, 1].min() >= 0.0
