"""The GPU 2-D step on a one-row rectangle strip (K = 4 face slots) against
the 1-D model of the oracle, compiled from the reference's shipped headers
when available: one GPU step from each state of a 60-step 1-D trajectory
lands on the next 1-D state (see test_strip_pin.py for why the strip
reduces exactly)."""
import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, mesh as meshmod
from zoomy_dmplex_b200.solver import Solver

from test_strip_pin import _oracle, _setup

pytestmark = pytest.mark.gpu


def test_gpu_strip_one_step_map_equals_1d():
    try:
        O.load(ref=True)
        ref = True
    except FileNotFoundError:
        ref = False
    x, q1, q2, p1, p2 = _setup()
    one = _oracle("sme1d_l0_malpasset", meshmod.interval(x), p1, ref=ref)
    g = Solver("sme2d_l0", meshmod.quad_strip(x), cases.default_settings(), p2)
    one.set_state(q1)
    t = 0.0
    worst = 0.0
    for k in range(60):
        a = one.get_state()
        dt = one.time()[1]
        g.set_state(np.concatenate([a, np.zeros((a.shape[0], 1))], axis=1), t)
        one.step(1)
        g.step(1, dts=np.array([dt]))
        t += dt
        b1, b2 = one.get_state(), g.get_state()
        for i in range(3):
            worst = max(worst, np.linalg.norm(b2[:, i] - b1[:, i]) / max(np.linalg.norm(b1[:, i]), 1e-300))
        assert np.abs(b2[:, 3]).max() <= 1e-14
    assert worst <= 1e-14, worst
