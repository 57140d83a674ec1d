import numpy as np

from zoomy_dmplex_b200 import mesh as M


def _closure(m):
    C = m.n_cells
    s = np.zeros((C, 2))
    for k in range(m.max_faces):
        f = m.cell_faces[:, k]
        sign = np.where(m.face_cells[f, 0] == np.arange(C), 1.0, -1.0)
        s += sign[:, None] * m.face_normal[f]
    return np.abs(s).max()


def test_jittered_square_geometry():
    m = M.jittered_square(30, seed=3)
    assert m.n_cells == 2 * 29 * 29
    assert abs(m.cell_volume.sum() - 1.0) < 1e-12
    assert (m.cell_volume > 0).all()
    assert _closure(m) < 1e-14                      # closed cells
    # normals point from support[0] to support[1] / outwards
    d = m.face_centroid - m.cell_centroid[m.face_cells[:, 0]]
    assert ((d * m.face_normal).sum(1) > 0).all()
    # Euler: F = C + V - 1 for a disc-like triangulation
    assert m.n_faces == m.n_cells + m.vertices.shape[0] - 1
    bnd = m.face_cells[:, 1] < 0
    assert (m.face_bc[bnd] == 0).all() and (m.face_bc[~bnd] == -1).all()
    assert abs(np.linalg.norm(m.face_normal[bnd], axis=1).sum() - 4.0) < 1e-12


def test_face_numbering_first_encounter():
    m = M.jittered_square(12, seed=0)
    # support[0] is the first cell that lists the face
    first = np.full(m.n_faces, -1)
    for c in range(m.n_cells):
        for f in m.cell_faces[c]:
            if first[f] < 0:
                first[f] = c
    assert (first == m.face_cells[:, 0]).all()
    # faces are numbered in first-encounter order
    order = [f for c in range(m.n_cells) for f in m.cell_faces[c]]
    seen = []
    for f in order:
        if f not in seen:
            seen.append(f)
    assert seen == list(range(m.n_faces))


def test_neighbours_cone_order():
    m = M.jittered_square(10, seed=1)
    nb = m.cell_nbrs()
    for c in range(m.n_cells):
        want = [int(m.face_cells[f, 1] if m.face_cells[f, 0] == c else m.face_cells[f, 0])
                for f in m.cell_faces[c]]
        want = [v for v in want if v >= 0]
        assert list(nb[c][: len(want)]) == want


def test_interval_and_msh_roundtrip(tmp_path):
    m = M.interval(np.linspace(0, 1, 11))
    assert m.n_cells == 10 and m.n_faces == 11 and m.dim == 1
    assert np.allclose(np.abs(m.face_normal[:, 0]), 1.0)
    m2 = M.jittered_square(8, seed=2)
    p = tmp_path / "m.msh"
    M.write_msh(str(p), m2)
    m3 = M.read_msh(str(p))
    assert m3.n_cells == m2.n_cells and np.allclose(m3.cell_volume.sum(), 1.0)


def test_mixed_triangles_and_quadrilaterals():
    """Ragged cells: -1 padded rows (triangles among quadrilaterals) have
    an empty face slot; the geometry is closed and consistently oriented,
    the numbering is first-encounter as for uniform meshes, and a gmsh file
    of the mesh reads back bit for bit."""
    m = M.mixed_square(10, seed=2)
    nv = (m.cells >= 0).sum(1)
    assert set(nv) == {3, 4} and m.max_faces == 4
    assert np.array_equal(m.cell_faces < 0, m.cells < 0)     # one empty slot per triangle
    assert abs(m.cell_volume.sum() - 1.0) < 1e-12 and (m.cell_volume > 0).all()
    C = m.n_cells
    s = np.zeros((C, 2))
    for k in range(m.max_faces):
        f = m.cell_faces[:, k]
        ok = f >= 0
        sign = np.where(m.face_cells[f[ok], 0] == np.arange(C)[ok], 1.0, -1.0)
        s[ok] += sign[:, None] * m.face_normal[f[ok]]
    assert np.abs(s).max() < 1e-14
    d = m.face_centroid - m.cell_centroid[m.face_cells[:, 0]]
    assert ((d * m.face_normal).sum(1) > 0).all()
    assert m.n_faces == C + m.vertices.shape[0] - 1                 # Euler, disc-like
    first = np.full(m.n_faces, -1)
    for c in range(C):
        for f in m.cell_faces[c]:
            if f >= 0 and first[f] < 0:
                first[f] = c
    assert (first == m.face_cells[:, 0]).all()
    fcs = m.cell_faces
    interior = (fcs >= 0) & (m.face_cells[np.maximum(fcs, 0), 1] >= 0)
    assert np.array_equal((m.cell_nbrs() >= 0).sum(1), interior.sum(1))


def test_mixed_mesh_gmsh_roundtrip(tmp_path):
    from zoomy_dmplex_b200 import caseio

    m = M.mixed_square(7, seed=4)
    p = str(tmp_path / "mixed.msh")
    caseio.write_gmsh(p, m, np.where(m.face_cells[:, 1] < 0, 1, 0), {1: "default"})
    r = caseio.read_gmsh(p)
    for a in ("cells", "cell_centroid", "cell_volume", "cell_faces", "face_cells", "face_centroid",
              "face_normal", "face_bc"):
        assert np.array_equal(getattr(m, a), getattr(r, a)), a
    v = str(tmp_path / "mixed.vtu")
    caseio.write_vtu(v, m, np.zeros((m.n_cells, 3)))
    d = caseio.read_vtu_cell_data(v)
    nv = (m.cells >= 0).sum(1)
    assert np.array_equal(d["offsets"], np.cumsum(nv))
    assert np.array_equal(d["types"], np.where(nv == 3, 5, 9))
    assert np.array_equal(d["connectivity"], m.cells[m.cells >= 0])


def test_pad_face_slots_keeps_the_mesh():
    """A triangle mesh taken to 4 face slots: empty slots added, geometry and
    numbering untouched, and the oracle step bit-identical."""
    import oracle_py as O
    from zoomy_dmplex_b200 import cases, models

    c = cases.level2(12)
    p = M.pad_face_slots(c.mesh, 4)
    assert p.max_faces == 4 and (p.cell_faces[:, 3] == -1).all() and (p.cells[:, 3] == -1).all()
    assert np.array_equal(p.cell_faces[:, :3], c.mesh.cell_faces)
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    out = []
    for m in (c.mesh, p):
        o = O.Oracle(c.model, m.as_abi_arrays(), c.settings.to_struct(), np.array(vals))
        o.set_state(c.q0)
        o.step(5)
        out.append(o.get_state())
    assert np.array_equal(out[0], out[1])
