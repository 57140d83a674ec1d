"""The partitioned GPU step (zoomy-dmplex_b200/partition.py): every part an
ordinary solver handle on its local mesh, the halo refreshed through
zsme_get_cells / zsme_set_cells after each step, the dt the minimum over the
parts -- against the undivided GPU run, bit for bit."""
import numpy as np
import pytest

from zoomy_dmplex_b200 import cases, partition as P
from zoomy_dmplex_b200.solver import Solver

from test_gpu_parity import params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nparts", [("l2", 2), ("l2", 4), ("l4", 3), ("mixed", 3)])
def test_partitioned_equals_undivided(name, nparts):
    c = {"l2": lambda: cases.level2(40), "l4": lambda: cases.roofline_l4(36),
         "mixed": lambda: cases.mixed_level2(30)}[name]()
    p = params(c.model, c.params)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    ps = P.PartitionedSolver(c.model, c.mesh, c.settings, p, nparts)
    ps.set_state(c.q0)
    assert ps.dt() == g.time()[1]
    for k in range(20):
        g.step(1)
        ps.step(1)
    assert ps.time() == g.time()[0]
    assert np.array_equal(ps.get_state(), g.get_state())


def test_cells_io_round_trip():
    c = cases.level2(20)
    g = Solver(c.model, c.mesh, c.settings, params(c.model, c.params))
    g.set_state(c.q0)
    ids = np.array([5, 0, 17, 3], dtype=np.int32)
    assert np.array_equal(g.get_cells(ids), g.get_state()[ids])
    q = g.get_state()
    new = q[ids] * 1.01
    g.set_cells(ids, new)
    q[ids] = new
    assert np.array_equal(g.get_state(), q)
    a = g.get_aux()
    g.set_state(q)                       # aux recomputed from the same state
    assert np.array_equal(g.get_aux()[ids], a[ids])
