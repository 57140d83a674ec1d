"""The library-free HDF5 reader behind caseio.load_state (the reference's
IOManager::LoadSolution reads dataset "state", IOManager.hpp:122-192):
round trips through the writer of the reference's generate_ic.py layout,
the component mask, shape checks, and a file written by the HDF5 library
itself (scipy's MATLAB 7.3 test file, when installed) read to the values
scipy's own tests expect."""
import os
import struct

import numpy as np
import pytest

from zoomy_dmplex_b200 import caseio, cases, hdf5


def test_state_round_trip_and_attributes(tmp_path):
    c = cases.level2(16)
    p = str(tmp_path / "ic.h5")
    hdf5.write_state(p, c.q0)
    a, attrs = hdf5.read_dataset(p)
    assert a.shape == (c.q0.size,) and a.dtype == np.float64
    assert int(attrs["num_cells"]) == c.mesh.n_cells and int(attrs["num_components"]) == c.q0.shape[1]
    assert np.array_equal(caseio.load_state(p), c.q0)
    assert np.array_equal(caseio.load_state(p, n_cells=c.mesh.n_cells, n_dof_q=8), c.q0)
    assert hdf5.list_root(p) == ["state"]


def test_mask_overlays_only_listed_components(tmp_path):
    c = cases.level2(12)
    loaded = c.q0 + 1.0
    p = str(tmp_path / "ic.hdf5")
    hdf5.write_state(p, loaded)
    q = caseio.overlay_state(c.q0, caseio.load_state(p), mask=[1, 3])
    assert np.array_equal(q[:, [1, 3]], loaded[:, [1, 3]])
    assert np.array_equal(q[:, [0, 2, 4, 5, 6, 7]], c.q0[:, [0, 2, 4, 5, 6, 7]])


def test_shape_errors_and_foreign_files(tmp_path):
    p = str(tmp_path / "ic.h5")
    hdf5.write_state(p, np.arange(12.0).reshape(4, 3))
    with pytest.raises(hdf5.HDF5Error, match="cells"):
        hdf5.read_state(p, n_cells=5)
    with pytest.raises(hdf5.HDF5Error, match="no object"):
        hdf5.read_dataset(p, "nothing")
    bad = str(tmp_path / "bad.h5")
    with open(bad, "wb") as f:
        f.write(b"not hdf5" * 20)
    with pytest.raises(hdf5.HDF5Error, match="signature"):
        hdf5.read_dataset(bad)


def test_big_endian_flat_state_without_attributes(tmp_path):
    """A flat dataset with no num_components attribute takes the model's
    n_dof_q; big-endian storage is converted."""
    p = str(tmp_path / "ic.h5")
    q = np.random.default_rng(1).standard_normal((10, 4))
    hdf5.write_state(p, q)
    raw = bytearray(open(p, "rb").read())
    # drop the attributes: a header with 4 messages (dataspace, type, fill, layout)
    f = hdf5._File(bytes(raw))
    a = f.resolve("state")
    hp = f.at(a)
    raw[hp + 2:hp + 4] = struct.pack("<H", 4)
    with open(p, "wb") as fh:
        fh.write(bytes(raw))
    assert np.array_equal(hdf5.read_state(p, n_dof_q=4), q)
    # the same values stored big endian
    f = hdf5._File(bytes(raw))
    (dpos,) = [r for mt, r, ms in f.messages(a) if mt == 0x03]
    (lpos,) = [r for mt, r, ms in f.messages(a) if mt == 0x08]
    raw[dpos + 1] |= 1
    da = f.at(f.addr(lpos + 2))
    raw[da:da + q.nbytes] = q.astype(">f8").tobytes()
    with open(p, "wb") as fh:
        fh.write(bytes(raw))
    assert np.array_equal(hdf5.read_state(p, n_dof_q=4), q)


MATLAB = os.path.join(os.path.dirname(np.__file__), "..", "scipy", "io", "matlab", "tests", "data",
                      "testhdf5_7.4_GLNX86.mat")


@pytest.mark.skipif(not os.path.exists(MATLAB), reason="scipy's HDF5 test file is not installed")
def test_reads_a_file_written_by_the_hdf5_library():
    """A 512-byte user block, superblock version 0, a version 2 layout
    message: MATLAB stores theta = pi/4 * [0, 1, ..., 8] there (scipy's
    test_mio expectation for 'testdouble')."""
    assert hdf5.list_root(MATLAB) == ["testdouble"]
    a, _ = hdf5.read_dataset(MATLAB, "testdouble")
    assert np.allclose(a.ravel(), np.pi / 4 * np.arange(9), rtol=0, atol=1e-15)
