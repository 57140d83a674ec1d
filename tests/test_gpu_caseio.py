"""The GPU step on meshes read from gmsh files with named boundaries:
boundary faces without a mapped tag carry no flux (TransportStep.hpp:496-500)
on both sides, per step against the oracle; snapshots of a GPU run."""
import os

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import caseio, cases, mesh as M
from zoomy_dmplex_b200.mesh import FACE_NO_CONDITION
from zoomy_dmplex_b200.solver import Solver

from test_caseio import SIDES, side_tags
from test_gpu_parity import TOL, errs, params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


def gmsh_case(tmp_path, tags_model):
    m = M.jittered_square(40, seed=3)
    p = str(tmp_path / "sq.msh")
    caseio.write_gmsh(p, m, side_tags(m), SIDES)
    r = caseio.read_gmsh(p, tags_model)
    x, y = r.cell_centroid[:, 0], r.cell_centroid[:, 1]
    b = 0.2 * np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / 0.01)
    h = 1.0 - b + 0.05 * np.exp(-((x - 0.3) ** 2 + (y - 0.3) ** 2) / 0.005)
    q = np.stack([b, h, 0.2 * h, 0.1 * h], axis=1)
    return r, q


def test_open_sides_per_step(tmp_path):
    m, q = gmsh_case(tmp_path, ["default"])
    assert caseio.boundary_counts(m)[FACE_NO_CONDITION] > 0
    s = cases.default_settings()
    p = params("sme2d_l0", dict(g=9.81, n_manning=0.0))
    g = Solver("sme2d_l0", m, s, p)
    o = O.Oracle("sme2d_l0", m.as_abi_arrays(), s.to_struct(), p)
    g.set_state(q)
    o.set_state(q)
    for k in range(40):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        e = errs(g.get_state(), o.get_state()).max()
        assert e <= TOL, "step %d: %g" % (k, e)


def test_snapshots_of_a_gpu_run(tmp_path):
    m, q = gmsh_case(tmp_path, ["default"])
    s = cases.default_settings(t_end=0.02)
    g = Solver("sme2d_l0", m, s, params("sme2d_l0", dict(g=9.81)))
    g.set_state(q)
    w = caseio.SnapshotWriter(str(tmp_path / "out"), "sol", t_end=0.02, snapshots=2)
    n = caseio.run_with_snapshots(g, m, w, 0.02)
    assert n > 0 and abs(g.time()[0] - 0.02) <= 1e-15
    assert [f for f, _ in w.log][0] == "sol-000.vtu" and len(w.log) == 3
    last = caseio.read_vtu_cell_data(os.path.join(str(tmp_path / "out"), w.log[-1][0]))
    assert np.array_equal(last["Q"], g.get_state()) and np.array_equal(last["Aux"], g.get_aux())
