"""The dual-number tangent-linear oracle against central finite differences
of the plain oracle (dt sequence frozen), on the adjoint case's physics: SME
level 1 with Manning friction, order 2, Green-Gauss, Vacuum + TVD limiting.

The discrete step is only piecewise smooth: the TVD ratio (q_max - q) / dq
has slope ~1/dq near extrema, the Newton loop may stop after 0 or 1
iterations (a jump of up to its 1e-8 tolerance), and max / |.| branches
switch.  Central differences with eps = 1e-6 therefore agree with the
tangent only while no such switch lies within eps of the trajectory: short
horizons with the limiter on, longer ones with it off, and smooth (sums of
Gaussians) rather than per-cell white-noise directions.  The tangent itself
is the exact derivative of the branch the run takes, which is what the
adjoint reproduces."""
import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, models


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals), names


def smooth_direction(mesh, rng, bumps=6):
    """A seeded random smooth field: a sum of Gaussians with random centres,
    widths and signed amplitudes."""
    x, y = mesh.cell_centroid[:, 0], mesh.cell_centroid[:, 1]
    d = np.zeros_like(x)
    for _ in range(bumps):
        cx, cy = rng.uniform(0, 1, 2)
        w = rng.uniform(0.02, 0.1)
        d += rng.standard_normal() * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / w)
    return d


def _tlm_vs_fd(n, nsteps, what, eps=1e-6, **settings):
    c = cases.adjoint_l1(n)
    for k, v in settings.items():
        setattr(c.settings, k, v)
    p, names = _params(c)
    st = c.settings.to_struct()
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st, p)
    o.set_state(c.q0)
    dts = []
    for _ in range(nsteps):
        dts.append(o.time()[1])
        o.step(1)
    dts = np.array(dts)
    dq = np.zeros_like(c.q0)
    dp = np.zeros_like(p)
    if what == "b":
        dq[:, 0] = smooth_direction(c.mesh, np.random.default_rng(5)) * 1e-2
    else:
        dp[names.index("n_manning")] = 1.0
    t = O.TangentOracle(c.model, c.mesh.as_abi_arrays(), st, p)
    t.set_state(c.q0)
    t.set_tangent(dq, dp)
    t.step(nsteps, dts=dts)
    tan = t.get_tangent()
    outs = []
    for sgn in (1, -1):
        o2 = O.Oracle(c.model, c.mesh.as_abi_arrays(), st, p + sgn * eps * dp)
        o2.set_state(c.q0 + sgn * eps * dq)
        o2.step(nsteps, dts=dts)
        outs.append(o2.get_state())
    fd = (outs[0] - outs[1]) / (2 * eps)
    assert np.linalg.norm(fd) > 0
    return np.linalg.norm(tan - fd) / np.linalg.norm(fd)


@pytest.mark.parametrize("what,tol", [("b", 1e-6),
                                      # the state's tangent in n is O(1e-4), so
                                      # rounding alone costs 1e-16 / 2e-6 / 1e-4
                                      # ~ 5e-7 of it
                                      ("manning", 1e-5)])
def test_tlm_matches_central_fd_limited(what, tol):
    rel = _tlm_vs_fd(16, 12, what)
    assert rel < tol, rel


def test_tlm_matches_central_fd_unlimited_long():
    rel = _tlm_vs_fd(40, 60, "b", limiter="none")
    assert rel < 1e-6, rel


def test_tlm_zero_direction_is_zero():
    c = cases.adjoint_l1(12)
    p, _ = _params(c)
    t = O.TangentOracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), p)
    t.set_state(c.q0)
    t.set_tangent(None, None)
    t.step(3)
    assert np.abs(t.get_tangent()).max() == 0.0
