"""Positivity variants on the GPU (libzsme.so through the C ABI) against the
oracle: the eta-well-balanced face states (prep_wb_kernel), the Zhang-Shu
CFL clamp, and MOOD's first-order override of troubled cells (mood_kernel),
per step and through the captured step graph.

Bar as for the plain step: per-step relative L2 and max error <= 1e-12; the
right-hand side (no Manning cbrt) is compared bit for bit.
"""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases
from zoomy_dmplex_b200.native import ZsmeError
from zoomy_dmplex_b200.solver import Solver

from test_gpu_parity import TOL, errs, params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


def pair(case, **kw):
    s = dataclasses.replace(case.settings, **kw)
    p = params(case.model, case.params)
    g = Solver(case.model, case.mesh, s, p)
    o = O.Oracle(case.model, case.mesh.as_abi_arrays(), s.to_struct(), p)
    g.set_state(case.q0)
    o.set_state(case.q0)
    return g, o


CASES = {
    "patch_l0": cases.wet_dry_patchwork(24),
    "patch_l1": cases.wet_dry_patchwork(24, seed=5, level=1),
    "l2": cases.level2(40),
    "l4": cases.roofline_l4(40),
    "mixed": cases.mixed_level2(24),
}


@pytest.mark.parametrize("pos", ["zhang_shu", "mood"])
@pytest.mark.parametrize("name", list(CASES))
def test_rhs_bitwise(name, pos):
    c = CASES[name]
    g, o = pair(c, positivity=pos)
    x = o.get_state()
    assert np.array_equal(g.rhs(x), o.rhs(x))


@pytest.mark.parametrize("pos", ["zhang_shu", "mood"])
@pytest.mark.parametrize("name", ["patch_l0", "patch_l1", "l2", "mixed"])
def test_trajectory_per_step(name, pos):
    """Free-running oracle; the GPU takes the oracle's dt each step."""
    c = CASES[name]
    g, o = pair(c, positivity=pos)
    assert abs(g.time()[1] - o.time()[1]) <= TOL * o.time()[1]   # CFL (clamped for zhang_shu)
    seen = 0
    for k in range(c.steps if name.startswith("patch") else 30):
        _, dt = o.time()
        m0 = o.mood_cells()
        o.step(1)
        g.step(1, dts=[dt])
        qg, qo = g.get_state(), o.get_state()
        e = errs(qg, qo).max()
        assert e <= TOL, "step %d: %g" % (k, e)
        d = g.sync(check=False)
        assert d.n_mood_cells == o.mood_cells() - m0, "step %d" % k
        seen += d.n_mood_cells
        assert qg[:, 1].min() >= 0.0
    if pos == "mood" and name == "patch_l0":
        assert seen > 0


def test_mood_graph_free_running():
    """The captured step (state copy + mood_kernel inside the graph), both
    sides choosing their own dt."""
    c = CASES["patch_l0"]
    g, o = pair(c, positivity="mood")
    g.step(c.steps)
    o.step(c.steps)
    d = g.sync(check=False)
    assert errs(g.get_state(), o.get_state()).max() <= TOL
    assert abs(g.time()[0] - o.time()[0]) <= TOL * o.time()[0]
    assert d.n_mood_cells > 0 and d.n_negative_depth == 0


def test_adjoint_rejects_positivity_variants():
    c = cases.adjoint_l1(16)
    g, _ = pair(c, positivity="zhang_shu")
    with pytest.raises(ZsmeError, match="positivity"):
        g.adjoint(2, [1], [0], [1], [0.0])
