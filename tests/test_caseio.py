"""Case I/O: gmsh 2.2 meshes with physical names mapped to model boundary
tags as the reference maps them (MeshConfigLoader.hpp:15-42,
VirtualSolver.hpp:391-411, 499-511), VTK snapshots with the .vtu.series
index (IOManager.hpp:33-79, 100-120, 346-360), and initial-state overlays
(IOManager.hpp:145-183)."""
import json
import os

import numpy as np
import pytest

from zoomy_dmplex_b200 import caseio, mesh as M
from zoomy_dmplex_b200.mesh import FACE_NO_CONDITION

SIDES = {1: "left", 2: "right", 3: "bottom", 4: "top"}


def side_tags(m):
    """Physical tag of each boundary face of a unit-square mesh by side."""
    x, y = m.face_centroid[:, 0], m.face_centroid[:, 1]
    bnd = m.face_cells[:, 1] < 0
    t = np.zeros(m.n_faces, dtype=np.int64)
    t[bnd & (x < 1e-12)] = 1
    t[bnd & (x > 1 - 1e-12)] = 2
    t[bnd & (y < 1e-12)] = 3
    t[bnd & (y > 1 - 1e-12)] = 4
    return t


def same_geometry(a, b):
    for k in ("cells", "cell_faces", "face_cells"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for k in ("cell_centroid", "cell_volume", "face_centroid", "face_normal"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_named_boundaries_triangles(tmp_path):
    m = M.jittered_square(7, seed=3)
    tags = side_tags(m)
    p = str(tmp_path / "sq.msh")
    caseio.write_gmsh(p, m, tags, SIDES)
    assert caseio.physical_names(p)["top"] == (1, 4)
    # model tags {"default"}: "default" takes tag 1 ("left"); the other sides have no condition
    r = caseio.read_gmsh(p, ["default"])
    same_geometry(r, m)
    bnd = r.face_cells[:, 1] < 0
    assert np.all(r.face_bc[bnd & (tags == 1)] == 0)
    assert np.all(r.face_bc[bnd & (tags != 1)] == FACE_NO_CONDITION)
    assert np.all(r.face_bc[~bnd] == -1)
    # a named model tag takes its own index
    r = caseio.read_gmsh(p, ["default", "top", "bottom"])
    assert np.all(r.face_bc[tags == 4] == 1) and np.all(r.face_bc[tags == 3] == 2)
    assert np.all(r.face_bc[tags == 2] == FACE_NO_CONDITION)
    # a model tag the file does not name is an error
    with pytest.raises(ValueError, match="exactly match"):
        caseio.read_gmsh(p, ["default", "inflow"])


def test_default_named_in_file_and_quads(tmp_path):
    n = 5
    s = np.linspace(0, 1, n + 1)
    X, Y = np.meshgrid(s, s, indexing="xy")
    v = np.stack([X.ravel(), Y.ravel()], 1)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    a = (j * (n + 1) + i).ravel()
    quads = np.stack([a, a + 1, a + n + 2, a + n + 1], 1)
    m = M.from_polygons(v, quads)
    tags = np.where(m.face_cells[:, 1] < 0, 7, 0)
    p = str(tmp_path / "q.msh")
    caseio.write_gmsh(p, m, tags, {7: "default"})
    r = caseio.read_gmsh(p)
    same_geometry(r, m)
    assert caseio.boundary_counts(r) == {0: 4 * n}


def test_interval_end_tags(tmp_path):
    m = M.interval(np.linspace(-1.5, 1.5, 31))
    x = m.face_centroid[:, 0]
    tags = np.where(x < -1.4, 1, np.where(x > 1.4, 2, 0))
    p = str(tmp_path / "i.msh")
    caseio.write_gmsh(p, m, tags, {1: "left", 2: "right"})
    r = caseio.read_gmsh(p)
    same_geometry(r, m)
    assert r.face_bc[np.argmin(x)] == 0 and r.face_bc[np.argmax(x)] == FACE_NO_CONDITION
    caseio.write_gmsh(p, m, tags, {1: "right", 2: "left"})
    r = caseio.read_gmsh(p, ["default", "left"])
    assert r.face_bc[np.argmin(x)] == 0 and r.face_bc[np.argmax(x)] == 1


def test_legacy_wrappers(tmp_path):
    m = M.jittered_square(6, seed=1)
    p = str(tmp_path / "w.msh")
    M.write_msh(p, m)
    r = M.read_msh(p)
    same_geometry(r, m)
    assert caseio.boundary_counts(r) == {0: int((m.face_cells[:, 1] < 0).sum())}


class _FakeSolver:
    def __init__(self, C, nq):
        self.t, self.C, self.nq = 0.0, C, nq

    def time(self):
        return self.t, 0.3

    def step(self, n=1):
        self.t = min(1.0, self.t + 0.3 * n)

    def get_state(self):
        return np.full((self.C, self.nq), self.t)

    def get_aux(self):
        return np.full((self.C, 1), 2 * self.t)


def test_snapshots_and_series(tmp_path):
    m = M.jittered_square(5, seed=0)
    w = caseio.SnapshotWriter(str(tmp_path / "out"), "sol", t_end=1.0, snapshots=4)
    g = _FakeSolver(m.n_cells, 4)
    n = caseio.run_with_snapshots(g, m, w, 1.0)
    # times 0, .3, .6, .9, 1.0 against next_snap 0, .25, .5, .75, 1.0
    assert n == 4 and [t for _, t in w.log] == pytest.approx([0.0, 0.3, 0.6, 0.9, 1.0], abs=1e-15)
    d = str(tmp_path / "out")
    assert sorted(os.listdir(d)) == ["sol-%03d.vtu" % i for i in range(5)] + ["sol.vtu.series"]
    txt = open(os.path.join(d, "sol.vtu.series")).read()
    assert '    { "name" : "sol-001.vtu", "time" : 3.000000e-01 },\n' in txt
    js = json.loads(txt)
    assert js["file-series-version"] == "1.0" and len(js["files"]) == 5
    cd = caseio.read_vtu_cell_data(os.path.join(d, "sol-002.vtu"))
    assert cd["Q"].shape == (m.n_cells, 4) and np.all(cd["Q"] == w.log[2][1]) and np.all(cd["Aux"] == 2 * w.log[2][1])
    assert np.array_equal(cd["connectivity"].reshape(-1, 3), m.cells)
    with pytest.raises(ValueError):
        caseio.SnapshotWriter(str(tmp_path / "x"), "s", 1.0, snapshots=0)


def test_initial_state_overlay(tmp_path):
    q = np.arange(12.0).reshape(3, 4)
    f = -np.arange(12.0).reshape(3, 4)
    np.save(tmp_path / "s.npy", f)
    np.savez(tmp_path / "s.npz", state=f.ravel())
    for p in ("s.npy", "s.npz"):
        loaded = caseio.load_state(str(tmp_path / p))
        assert np.array_equal(caseio.overlay_state(q, loaded), f)
        o = caseio.overlay_state(q, loaded, [1, 3, 9])
        assert np.array_equal(o[:, [0, 2]], q[:, [0, 2]]) and np.array_equal(o[:, [1, 3]], f[:, [1, 3]])
    # HDF5 in the reference's layout (hdf5.write_state, as its generate_ic.py writes it)
    from zoomy_dmplex_b200 import hdf5

    hdf5.write_state(str(tmp_path / "s.h5"), f)
    loaded = caseio.load_state(str(tmp_path / "s.h5"))
    assert np.array_equal(caseio.overlay_state(q, loaded, [1, 3])[:, [1, 3]], f[:, [1, 3]])
    with pytest.raises(ValueError, match="h5"):
        caseio.load_state(str(tmp_path / "s.txt"))


@pytest.mark.skipif(not os.environ.get("ZSME_GMSH_DIR"), reason="ZSME_GMSH_DIR (a directory of gmsh cases) unset")
def test_external_gmsh_cases():
    """Optional: the bump cases of a case directory (bump_1d.msh: 200
    segments, ends "left"/"right"; bump_2d.msh: 120 x 8 quadrilaterals,
    sides left/right/bottom/top) read with the model tags {"default"}."""
    d = os.environ["ZSME_GMSH_DIR"]
    m1 = caseio.read_gmsh(os.path.join(d, "bump_1d.msh"))
    assert m1.dim == 1 and m1.n_cells == 200
    assert caseio.boundary_counts(m1) == {FACE_NO_CONDITION: 1, 0: 1}
    m2 = caseio.read_gmsh(os.path.join(d, "bump_2d.msh"))
    assert m2.dim == 2 and m2.n_cells == 960 and m2.cells.shape[1] == 4
    assert caseio.boundary_counts(m2) == {FACE_NO_CONDITION: 248, 0: 8}
    assert np.isclose(m2.cell_volume.sum(), np.ptp(m2.vertices[:, 0]) * np.ptp(m2.vertices[:, 1]))
