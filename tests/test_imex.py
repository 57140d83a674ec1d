"""The IMEX time integration on the oracle (the reference's IMEX strategy,
SolverStrategies.hpp:62-128: PETSc's additive Runge-Kutta scheme "2e" with
the transport explicit and the source implicit per cell), restated at the
step's CFL dt without PETSc's step-size control:

* the tableau (zoomy-dmplex_b200/csrc/imex_tableau.h, parsed here) meets the
  order conditions of a second-order additive scheme;
* on a smooth problem the error falls at second order in dt, against first
  order for the operator splitting of the same first-order space scheme;
* mass is conserved to rounding with reflective walls, and a lake at rest
  stays at rest;
* a stiff Navier-slip source (friction time far below the CFL dt) stays
  bounded, as an implicit source must.
"""
import dataclasses
import os
import re

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _tableau():
    src = open(os.path.join(ROOT, "zoomy-dmplex_b200", "csrc", "imex_tableau.h")).read()
    env = {}
    for name, expr in re.findall(r"constexpr double (\w+) = ([^;]+);", src):
        env[name] = eval(expr, {}, dict(env))
    return env


def test_tableau_order_conditions():
    k = _tableau()
    g = k["gamma"]
    A = np.array([[0, 0, 0], [k["a10"], 0, 0], [k["a20"], k["a21"], 0]])
    At = np.array([[0, 0, 0], [k["t10"], g, 0], [k["t20"], k["t21"], g]])
    b = np.array([k["b0"], k["b1"], k["b2"]])
    c = np.array([0.0, k["c1"], k["c2"]])
    for M in (A, At):
        assert np.allclose(M.sum(axis=1), c, atol=1e-15)      # row sums are the stage times
    assert abs(b.sum() - 1) < 1e-15
    assert abs(b @ c - 0.5) < 1e-15                          # second order, both parts and coupled
    assert np.allclose(b, At[-1], atol=0)                    # stiffly accurate implicit part
    assert abs(g - (1 - 1 / np.sqrt(2))) < 1e-16


def _params(c):
    names, vals = models.parameter_table(c.model)
    for kk, v in c.params.items():
        vals[names.index(kk)] = v
    return np.array(vals)


def _run(c, p, dt, n, **kw):
    st = dataclasses.replace(c.settings, **kw)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), p)
    o.set_state(c.q0)
    o.step(n, dts=np.full(n, dt))
    return o


def test_second_order_in_time():
    O.set_threads(0)
    c = cases.level2(20)
    p = _params(c)
    T = 0.02
    ref = _run(c, p, T / 320, 320, time_integration="imex", reconstruction_order=1).get_state()
    err = {}
    for ti in ("imex", "splitting"):
        err[ti] = [np.linalg.norm(_run(c, p, T / k, k, time_integration=ti, reconstruction_order=1).get_state() - ref)
                   for k in (20, 40, 80)]
    rate_imex = np.log2(err["imex"][1] / err["imex"][2])
    rate_split = np.log2(err["splitting"][1] / err["splitting"][2])
    assert 1.8 < rate_imex < 2.6, err
    assert 0.8 < rate_split < 1.3, err
    assert err["imex"][2] < 1e-3 * err["splitting"][2]


def test_mass_and_lake_at_rest():
    c = cases.level2(20)
    p = _params(c)
    o = _run(c, p, 2e-4, 30, time_integration="imex")
    q = o.get_state()
    vol = c.mesh.cell_volume
    assert abs((q[:, 1] * vol).sum() - (c.q0[:, 1] * vol).sum()) < 1e-13
    assert q[:, 1].min() > 0
    rest = dataclasses.replace(c)
    rest.q0 = c.q0.copy()
    rest.q0[:, 1] = 1.0 - rest.q0[:, 0]
    rest.q0[:, 2:] = 0.0
    o = _run(rest, p, 2e-4, 20, time_integration="imex", reconstruction_order=1)
    q = o.get_state()
    assert np.abs(q[:, 0] + q[:, 1] - 1).max() < 1e-14 and np.abs(q[:, 2:]).max() < 1e-14


def test_stiff_source_stays_bounded():
    """Navier slip with slip length 1e-5 and viscosity 0.1: the friction
    rate (2i+1) nu / lambda per unit depth is about 1e4 per second, while the
    CFL step is of order 1e-3 s; the implicit stages damp the moments instead
    of blowing up."""
    c = cases.level2(20)
    names, _ = models.parameter_table(c.model)
    p = _params(c)
    p[names.index("lambda")] = 1e-5
    p[names.index("nu")] = 1e-1
    st = dataclasses.replace(c.settings, time_integration="imex")
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), p)
    o.set_state(c.q0)
    o.step(40)
    q = o.get_state()
    assert np.all(np.isfinite(q)) and q[:, 1].min() > 0
    assert np.abs(q[:, 2:]).max() < np.abs(c.q0[:, 2:]).max()


def test_unknown_strategy_is_rejected():
    c = cases.level2(8)
    with pytest.raises(ValueError, match="implicit"):
        dataclasses.replace(c.settings, time_integration="rosenbrock").to_struct()
