"""Algorithmic FP64 operation counts behind the bench's FP64 roofline.

The oracle instantiated on an operation-counting scalar (oracle/flopcount.h)
counts the +, -, *, /, sqrt, cbrt and pow of the reference step per phase
(prep, face, gather, finalize).  These tests recount the per-unit figures
the bench uses (bench.FP64_FLOPS), check that counting does not change the
arithmetic, and that the phases are attributed as the kernels split the
work.
"""
import dataclasses

import numpy as np
import pytest

import bench
import oracle_py as O
from zoomy_dmplex_b200 import cases, models

CONFIG_CASE = {"sme2d_l4": cases.roofline_l4, "sme2d_l2": cases.level2, "sme2d_l0": cases.plain_l0,
               "sme2d_l1": cases.adjoint_l1}


def params(case):
    names, vals = models.parameter_table(case.model)
    for k, v in case.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def count(case, settings=None, steps=2):
    st = settings or case.settings
    return O.flop_counts(case.model, case.mesh.as_abi_arrays(), st.to_struct(), params(case), case.q0, steps=steps)


@pytest.mark.parametrize("model", sorted(bench.FP64_FLOPS))
def test_table_recounts(model):
    c = CONFIG_CASE[model](40)
    r = count(c)
    tot = {k: sum(v.values()) for k, v in r.items()}
    C, F, s = c.mesh.n_cells, c.mesh.n_faces, c.settings.ssp_stages
    got = {"prep": tot["prep"] / (C * 2 * s), "flux": tot["face"] / (F * 2 * s),
           "gather": tot["gather"] / (C * 2 * s), "finalize": tot["final"] / (C * 2)}
    for k, v in bench.FP64_FLOPS[model].items():
        assert got[k] == pytest.approx(v, abs=1e-3), k
    assert bench.fp64_flops_per_cell_step(model, C, F, s) == pytest.approx(sum(tot.values()) / (C * 2), rel=1e-6)


def test_counting_keeps_the_arithmetic():
    """The counting instance's state after the steps is the plain oracle's,
    bit for bit (the counted scalar rounds as a double)."""
    import ctypes as ct

    from zoomy_dmplex_b200 import native

    c = cases.level2(24)
    lib = O.load()
    keep = native.make_mesh_struct(c.mesh.as_abi_arrays())
    st = c.settings.to_struct()
    p = np.ascontiguousarray(params(c))
    h = ct.c_void_p()
    assert lib.oracle_create_counting(c.model.encode(), ct.addressof(keep[0]), ct.addressof(st),
                                      O._p(p), ct.byref(h)) == 0
    q = np.ascontiguousarray(c.q0)
    lib.oracle_set_state(h, O._p(q), 0.0)
    lib.oracle_step(h, 3)
    out = np.zeros_like(q)
    lib.oracle_get_state(h, O._p(out))
    lib.oracle_destroy(h)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st, p)
    o.set_state(c.q0)
    o.step(3)
    assert np.array_equal(out, o.get_state())


def test_face_phase_independent_of_reconstruction():
    """Face work (face aux, flux, fluctuations, wall ghosts, area products)
    is straight-line model code: per right-hand-side evaluation the same
    count at order 1 (one Euler evaluation per step) and order 2 (s stage
    evaluations), the reconstruction being charged to prep."""
    c = cases.level2(24)
    s = c.settings.ssp_stages
    r1 = count(c, dataclasses.replace(c.settings, reconstruction_order=1), steps=1)
    r2 = count(c, steps=1)
    assert {k: s * v for k, v in r1["face"].items()} == r2["face"]
    assert sum(r2["prep"].values()) > 2 * s * sum(r1["prep"].values())
