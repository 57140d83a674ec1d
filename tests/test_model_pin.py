"""The generated model plugin vs the reference's own shipped generated
headers (1-D SME level 0): golden outputs of the reference's Model.H /
Numerics.H (tests/golden/ref1d_pointwise.npz, made by make_golden.py from
the reference compiled in oracle/_ref) against this repository's generator
output for the same model (models/sme1d_l0_malpasset)."""
import os

import numpy as np
import pytest

import oracle_py as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "ref1d_pointwise.npz"))

# Rounding-level tolerance; the solver-side finite-difference dAux/dQ
# (h = 1e-7 (|q|+1e-7)) amplifies last-bit differences of hinv by ~1/h.
TOL = {"aux_jacobian": 1e-6}


@pytest.mark.parametrize("fn", list(O.FN))
def test_generated_matches_reference_header(fn):
    X = GOLDEN["inputs"]
    ref = GOLDEN[fn]
    tol = TOL.get(fn, 1e-13)
    for r, want in zip(X, ref):
        qL, qR, aL, aR, p, nx, s = r[0:3], r[3:6], r[6:10], r[10:14], r[14:19], r[19], r[20]
        got = O.pointwise("sme1d_l0_malpasset", fn, qL, aL, p, np.array([nx, 0, 0]), qR, aR, s=s)
        assert got.shape == want.shape
        err = np.abs(got - want) / np.maximum(1.0, np.abs(want))
        assert np.all(np.isfinite(got) == np.isfinite(want))
        assert np.nanmax(np.where(np.isfinite(want), err, 0.0)) <= tol, (fn, r, got, want)


@pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="reference build (oracle/_ref) absent")
def test_oracle_step_with_reference_header():
    """The whole oracle step instantiated with the reference's header vs with
    the generated one, on a 1-D mesh (transport + source + dt)."""
    from zoomy_dmplex_b200 import mesh as M, cases
    m = M.interval(np.linspace(-1.5, 1.5, 121))
    x = m.cell_centroid[:, 0]
    b = 0.2 * np.exp(-x ** 2 / 0.05)
    h = 1.0 - b + 0.1 * np.exp(-(x + 0.5) ** 2 / 0.01)
    q = np.stack([b, h, 0.3 * h], axis=1)
    p = np.array([9.81, 1.0, 1.0, 0.2, 0.01])
    st = cases.default_settings().to_struct()
    outs = []
    for model in ("ref1d", "sme1d_l0_malpasset"):
        o = O.Oracle(model, m.as_abi_arrays(), st, p, ref=True)
        o.set_state(q)
        o.step(50)
        outs.append(o.get_state())
    rel = np.linalg.norm(outs[0] - outs[1]) / np.linalg.norm(outs[0])
    assert rel < 1e-12
