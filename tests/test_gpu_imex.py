"""The IMEX time integration on the GPU (imex_kernels.cuh: explicit
transport right-hand sides from the step kernels in MODE_RHS, implicit
source stages solved per cell, additive Runge-Kutta 2E) against the
oracle's restatement: every step bit for bit with the oracle's dt imposed,
free running on the CUDA graph, at both reconstruction orders, on the 1-D
model and in an ensemble; the adjoint refuses it."""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, native
from zoomy_dmplex_b200.solver import BatchSolver, Solver

from test_gpu_parity import params, case_1d

pytestmark = pytest.mark.gpu


def _pair(c, **kw):
    st = dataclasses.replace(c.settings, time_integration="imex", **kw)
    p = params(c.model, c.params)
    g = Solver(c.model, c.mesh, st, p)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), p)
    g.set_state(c.q0)
    o.set_state(c.q0)
    return g, o


@pytest.mark.parametrize("make,order,steps", [(lambda: cases.level2(30), 2, 30), (lambda: cases.level2(30), 1, 30),
                                              (lambda: cases.roofline_l4(24), 2, 15), (case_1d, 2, 40),
                                              (lambda: cases.mixed_level2(16), 2, 20)])
def test_imex_per_step_bitwise(make, order, steps):
    O.set_threads(0)
    c = make()
    g, o = _pair(c, reconstruction_order=order)
    for k in range(steps):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        assert np.array_equal(g.get_state(), o.get_state()), "step %d" % (k + 1)
    assert np.array_equal(g.get_aux(), o.get_aux())
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0


def test_imex_free_running_graph():
    c = cases.level2(30)
    g, o = _pair(c)
    g.step(25)
    o.step(25)
    assert g.time() == o.time()
    assert np.array_equal(g.get_state(), o.get_state())
    g.set_profiling(True)
    g.step(2)
    g.sync()
    n = sum(v[1] for v in g.read_profile().values())
    g.set_profiling(False)
    assert n > 0


def test_imex_ensemble_equals_loop():
    members = cases.ensemble(4, seed=11, side_range=(12, 30), processes=1)
    st = dataclasses.replace(members[0].settings, time_integration="imex")
    b = BatchSolver(members[0].model, [m.mesh for m in members], st, [params(m.model, m.params) for m in members])
    for i, m in enumerate(members):
        b.set_state(i, m.q0)
    b.step(15)
    for i, m in enumerate(members):
        g = Solver(m.model, m.mesh, st, params(m.model, m.params))
        g.set_state(m.q0)
        g.step(15)
        assert np.array_equal(b.get_state(i), g.get_state()), i
        assert b.time(i) == g.time()


def test_adjoint_refuses_imex():
    c = cases.adjoint_l1(12)
    g, _ = _pair(c)
    with pytest.raises(native.ZsmeError, match="splitting"):
        g.adjoint(3, [1], [0], [1], [1.0])
