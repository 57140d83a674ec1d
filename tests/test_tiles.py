"""Host-side tiling of the fused face + gather kernel (zsme_mesh_tiles, no
device needed): the tiles' own face ranges cover every face once, each
tile evaluates at most tile_faces faces, every cell-face incidence that
carries a flux is addressed, and the only repeated work is the incoming
faces (interior faces between two tiles), which shrink as tiles grow and
vanish for a single tile."""
import numpy as np
import pytest

from zoomy_dmplex_b200 import cases, mesh as meshmod, native


def _flux_slots(m):
    fc = m.face_cells
    interior = int(np.sum(fc[:, 1] >= 0))
    bnd = fc[:, 1] < 0
    with_condition = int(np.sum(bnd & (m.face_bc >= 0)))
    return interior, 2 * interior + with_condition


@pytest.mark.parametrize("make", [lambda: cases.level2(40), lambda: cases.mixed_level2(16),
                                  lambda: cases.plain_l0(30)])
@pytest.mark.parametrize("tile_faces", [64, 128, 256, 1024])
def test_tiles_cover_faces(make, tile_faces):
    c = make()
    st = native.mesh_tiles(c.mesh, tile_faces)
    interior, slots = _flux_slots(c.mesh)
    assert st["covered"] == c.mesh.n_faces
    assert st["max_faces"] <= tile_faces
    assert st["flux_slots"] == slots
    assert 0 <= st["incoming"] <= interior
    assert (st["incoming"] == 0) == (st["tiles"] == 1)
    assert st["tiles"] >= c.mesh.n_faces / tile_faces


def test_tiles_shrink_redundancy_and_one_tile_has_none():
    c = cases.level2(40)
    inc = [native.mesh_tiles(c.mesh, t)["incoming"] for t in (64, 128, 256, 512)]
    assert inc == sorted(inc, reverse=True)
    small = cases.level2(12)
    st = native.mesh_tiles(small.mesh, 1024)
    assert small.mesh.n_faces <= 1024 and st["tiles"] == 1 and st["incoming"] == 0


def test_tiles_on_a_1d_mesh_and_bad_sizes():
    m = meshmod.interval(np.linspace(0.0, 1.0, 101))
    st = native.mesh_tiles(m, 64)
    assert st["covered"] == m.n_faces and st["max_faces"] <= 64
    # a tile must hold at least two cells' faces
    with pytest.raises(native.ZsmeError):
        native.mesh_tiles(m, 3)
