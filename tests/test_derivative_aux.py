"""RefreshDerivativeAux on the oracle (TransportStep.hpp:161-202,
UserFunctions.H:60-112): with solver.refresh_derivative_aux on (the
reference's default) every state update first refills the plugin's
derivative aux slots -- for the 1-D level-0 model dq0/dx, dh/dx, db/dx --
with the Green-Gauss derivative of the state, zero Neumann at the ends.
Checked against a plain restatement of that face loop, against the
reference's own shipped header (whose field-level update_aux_variables
requests the same derivatives), and for not touching the state."""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, mesh as meshmod, models


def _setup(n=160):
    x = np.linspace(-1.0, 2.0, n + 1) ** 3 / 4.0 + np.linspace(-1.0, 2.0, n + 1)   # uneven cells
    xc = 0.5 * (x[:-1] + x[1:])
    b = 0.2 * np.exp(-(xc - 0.5) ** 2 / 0.05)
    h = 1.0 - b + 0.05 * np.exp(-(xc - 0.2) ** 2 / 0.01)
    q = np.stack([b, h, 0.3 * h], axis=1)
    names, vals = models.parameter_table("sme1d_l0_malpasset")
    return meshmod.interval(x), q, np.array(vals, float)


def _gg_derivative(m, s):
    """compute_derivative's face loop, face by face in increasing face id."""
    g = np.zeros(m.n_cells)
    fc, fn = m.face_cells, m.face_normal
    for f in range(m.n_faces):
        a, b = fc[f]
        if b >= 0:
            v = (0.5 * (s[a] + s[b])) * fn[f, 0]
            g[a] += v
            g[b] -= v
        else:
            g[a] += s[a] * fn[f, 0]
    vol = m.cell_volume
    return np.where(vol > 0, g / np.where(vol > 0, vol, 1.0), 0.0)


def _oracle(m, p, refresh=True, ref=False):
    st = dataclasses.replace(cases.default_settings(), refresh_derivative_aux=refresh)
    return O.Oracle("sme1d_l0_malpasset", m.as_abi_arrays(), st.to_struct(), p, ref=ref)


def test_refresh_fills_green_gauss_derivatives():
    m, q, p = _setup()
    o = _oracle(m, p)
    o.set_state(q)
    o.step(7)
    s, a = o.get_state(), o.get_aux()
    for slot, comp in ((0, 2), (1, 1), (2, 0)):
        assert np.array_equal(a[:, slot], _gg_derivative(m, s[:, comp])), slot
    assert np.abs(a[:, 1]).max() > 0.1          # the hump's slope is there


def test_refresh_off_leaves_slots_and_state_unchanged():
    m, q, p = _setup()
    on, off = _oracle(m, p, True), _oracle(m, p, False)
    for o in (on, off):
        o.set_state(q)
        o.step(7)
    assert np.array_equal(on.get_state(), off.get_state())
    assert np.all(off.get_aux()[:, :3] == 0.0)
    assert np.array_equal(on.get_aux()[:, 3], off.get_aux()[:, 3])


def test_refresh_matches_the_reference_header():
    try:
        O.load(ref=True)
    except FileNotFoundError:
        pytest.skip("the reference-header oracle is not built (needs the reference sources)")
    m, q, p = _setup()
    ours, theirs = _oracle(m, p), _oracle(m, p, ref=True)
    for o in (ours, theirs):
        o.set_state(q)
        o.step(7)
    assert np.array_equal(ours.get_aux()[:, :3], theirs.get_aux()[:, :3])
    assert np.abs(theirs.get_aux()[:, :3]).max() > 0.0
