"""The batched ensemble (one handle, every launch covers all instances)
against looping the plain single-instance solver per instance, and against
the oracle.  Bar: the same per-variable 1e-12 as the plain path; with the
same kernels and per-instance CFL minima the results are bit-identical."""
import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models
from zoomy_dmplex_b200.solver import BatchSolver, Solver

pytestmark = pytest.mark.gpu


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


@pytest.fixture(scope="module")
def members():
    return cases.ensemble(6, seed=11, side_range=(12, 40), processes=1)


def test_batch_equals_per_instance_loop(members):
    st = members[0].settings
    b = BatchSolver(members[0].model, [c.mesh for c in members], st, [_params(c) for c in members])
    for i, c in enumerate(members):
        b.set_state(i, c.q0)
    b.step(30)
    d = b.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0
    for i, c in enumerate(members):
        g = Solver(c.model, c.mesh, st, _params(c))
        g.set_state(c.q0)
        g.step(30)
        assert np.array_equal(b.get_state(i), g.get_state()), i
        assert b.time(i) == g.time()


def test_batch_member_vs_oracle(members):
    c = members[2]
    st = c.settings
    b = BatchSolver(c.model, [m.mesh for m in members], st, [_params(m) for m in members])
    for i, m in enumerate(members):
        b.set_state(i, m.q0)
    O.set_threads(0)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), _params(c))
    o.set_state(c.q0)
    b.step(20)
    o.step(20)
    a, r = b.get_state(2), o.get_state()
    assert np.linalg.norm(a - r) <= 1e-12 * np.linalg.norm(r)
    assert abs(b.time(2)[0] - o.time()[0]) <= 1e-12 * o.time()[0]


def test_instances_have_own_dt(members):
    st = members[0].settings
    b = BatchSolver(members[0].model, [c.mesh for c in members], st, [_params(c) for c in members])
    for i, c in enumerate(members):
        b.set_state(i, c.q0)
    dts = [b.time(i)[1] for i in range(len(members))]
    assert len(set(dts)) > 1


def test_batch_rejects_single_instance_calls(members):
    from zoomy_dmplex_b200 import native
    st = members[0].settings
    b = BatchSolver(members[0].model, [c.mesh for c in members[:2]], st, [_params(c) for c in members[:2]])
    q = np.zeros((members[0].mesh.n_cells, b.nq))
    with pytest.raises(native.ZsmeError):
        native.check(b.lib.zsme_set_state(b.h, q.ctypes.data_as(native.ct.POINTER(native.ct.c_double)), 0.0))


def test_batch_mixes_triangle_and_quadrilateral_meshes():
    """Instances with different face-slot counts in one ensemble: triangle
    meshes get empty slots beside mixed triangle/quadrilateral meshes, and
    every instance ends bit-identical to its own plain solve."""
    members = [cases.level2(14, seed=3), cases.mixed_level2(12, seed=4), cases.level2(18, seed=5)]
    st = members[0].settings
    b = BatchSolver("sme2d_l2", [c.mesh for c in members], st, [_params(c) for c in members])
    for i, c in enumerate(members):
        b.set_state(i, c.q0)
    b.step(25)
    for i, c in enumerate(members):
        g = Solver(c.model, c.mesh, st, _params(c))
        g.set_state(c.q0)
        g.step(25)
        assert np.array_equal(b.get_state(i), g.get_state()), i
        assert b.time(i) == g.time()


def test_config3_members_batch_equals_loop():
    """The first 64 members of configuration 3's ensemble as specified (grid
    sides log-uniform in [40, 400], their own bumps, humps and CFL dt): one
    batched handle against one plain solver per member, 20 steps, every
    member bit-identical in state and time."""
    members = cases.ensemble(64)
    sides = [cases.ensemble_side(i) for i in range(64)]
    assert min(sides) < 80 and max(sides) > 250
    st = members[0].settings
    b = BatchSolver(members[0].model, [c.mesh for c in members], st, [_params(c) for c in members])
    for i, c in enumerate(members):
        b.set_state(i, c.q0)
    b.step(20)
    d = b.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0
    for i, c in enumerate(members):
        g = Solver(c.model, c.mesh, st, _params(c))
        g.set_state(c.q0)
        g.step(20)
        assert np.array_equal(b.get_state(i), g.get_state()), i
        assert b.time(i) == g.time(), i
        g.close()
