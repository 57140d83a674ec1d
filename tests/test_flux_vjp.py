"""The generated reverse-mode face derivative (numerical_flux_fluct_vjp,
printed by models/gen_sme.py) against the dual-number Jacobian of
numerical_flux and numerical_fluctuations, on random faces including the
kinks the adjoint meets: equal bed heights (the max(bL, bR) tie), a dry side,
a star depth of exactly zero, identical states."""
import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import models

MODELS = ["sme2d_l0", "sme2d_l1", "sme2d_l2", "sme2d_l4"]


def test_reference_style_header_has_none():
    """The 1-D model mirrors the reference's shipped header, which has no
    face VJP: the adjoint differentiates it with dual numbers."""
    q = np.array([0.1, 1.0, 0.2])
    assert O.flux_vjp("sme1d_l0_malpasset", q, q, np.ones(5), np.array([1.0, 0, 0]), np.ones(9)) is None


@pytest.mark.parametrize("model", MODELS)
def test_vjp_equals_dual_jacobian_contraction(model):
    names, vals = models.parameter_table(model)
    p = np.array(vals)
    nq = models.constants(model)["n_dof_q"]
    two_d = model.startswith("sme2d")
    rng = np.random.default_rng(nq)
    worst = 0.0
    for trial in range(400):
        kind = trial % 5
        qL, qR = np.zeros(nq), np.zeros(nq)
        qL[0], qR[0] = rng.uniform(0, 0.3, 2)
        if kind == 1:
            qR[0] = qL[0]
        qL[1], qR[1] = rng.uniform(0.0, 2.0, 2)
        if kind == 2:
            qL[1] = 0.0
        qL[2:] = rng.normal(0, 1, nq - 2) * qL[1]
        qR[2:] = rng.normal(0, 1, nq - 2) * qR[1]
        if kind == 3:       # star depth zero on the left: b_L + h_L < b_R
            qL[0], qL[1], qR[0] = 0.0, 1e-3, 0.5
        if kind == 4:
            qR = qL.copy()
        th = rng.uniform(0, 2 * np.pi)
        n = np.array([np.cos(th), np.sin(th), 0.0]) if two_d else np.array([1.0, 0.0, 0.0])
        w = rng.normal(size=3 * nq)
        ref = w @ O.face_jacobian(model, qL, qR, p, n)
        g = O.flux_vjp(model, qL, qR, p, n, w)
        assert g is not None and np.all(np.isfinite(g))
        worst = max(worst, np.abs(g - ref).max() / max(1.0, np.abs(ref).max()))
    assert worst <= 1e-13, worst
