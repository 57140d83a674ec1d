"""The fully implicit strategy on the oracle (SolverStrategies.hpp:133-195:
TSBDF order 2 on F(t, X, Xdot) = Xdot - S(X) - R(X), Newton with a
matrix-free Jacobian, the matrix of ModularSolver::FormImplicitJacobian as
the preconditioner's source), restated without PETSc:

* the residual equals Xdot - S - R assembled from the oracle's FormRHS and a
  pointwise restatement of the implicit source, bit for bit;
* the assembled matrix equals a plain restatement of FormImplicitJacobian
  built from pointwise plugin calls (forward differences of each face's
  flux and fluctuations, the source blocks, the assembly order), bit for
  bit, and at first order in space it is the Jacobian of F itself;
* BDF2 converges at second order in dt; a lake at rest stays at rest; mass
  is kept to the Newton tolerance; a stiff source at a large dt stays
  bounded;
* where the limited second-order residual is not differentiable (the TVD
  limiter's shared alpha switches under any perturbation of a flat field)
  Newton fails and the step leaves state and time as they were.
"""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, mesh as meshmod, models


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def _oracle(c, **kw):
    st = dataclasses.replace(c.settings, time_integration="implicit", **kw)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), _params(c))
    o.set_state(c.q0)
    return o


def _case_1d():
    x = np.linspace(-1.5, 1.5, 61)
    m = meshmod.interval(x)
    xc = m.cell_centroid[:, 0]
    b = 0.2 * np.exp(-xc ** 2 / 0.05)
    h = 1.0 - b + 0.1 * np.exp(-(xc + 0.5) ** 2 / 0.01)
    q = np.stack([b, h, 0.3 * h], axis=1)
    return cases.Case("1d", "sme1d_l0_malpasset", m, q, cases.default_settings(),
                      dict(g=9.81, rho=1.0, nu=1.0, lambda_s=0.2, e_x=0.01), 20)


CASES = {"l2": lambda: cases.level2(5), "1d": _case_1d, "mixed": lambda: cases.mixed_level2(4),
         "l0": lambda: cases.plain_l0(5)}


def _perturbed(c, seed=3):
    rng = np.random.default_rng(seed)
    x = c.q0.copy()
    x[:, 2:] += 0.05 * rng.standard_normal(x[:, 2:].shape) * x[:, 1:2]
    return x


def _pw(model, fn, qL, aL, p, n=None, qR=None, aR=None):
    return O.pointwise(model, fn, qL, aL, p, n=n, qR=qR, aR=aR)


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("order", [1, 2])
def test_residual_is_xdot_minus_source_minus_rhs(name, order):
    """IFunctionWrapper: F = Xdot, F += -S (AddImplicitSourceToResidual: the
    plugin's source at the clamped state, nothing where the depth is below
    1e-6), F += -R (FormRHS)."""
    c = CASES[name]()
    o = _oracle(c, reconstruction_order=order)
    x = _perturbed(c)
    xdot = np.random.default_rng(1).standard_normal(x.shape)
    f = o.implicit_function(x, xdot, t=0.3)
    R = o.rhs(x, t=0.3)
    p = _params(c)
    a0 = o.get_aux()                      # the aux the source starts from
    S = np.zeros_like(x)
    for k in range(c.mesh.n_cells):
        q = _pw(c.model, "update_variables", x[k], a0[k], p)
        a = _pw(c.model, "update_aux_variables", q, a0[k], p)
        if x.shape[1] > 1 and q[1] < 1e-6:
            continue
        S[k] = _pw(c.model, "source", q, a, p)
    assert np.array_equal(f, (xdot - S) - R)


def _restated_matrix(c, x, a_shift, p, aux0):
    """FormImplicitJacobian (ModularSolver.hpp:238-371) in numpy over
    pointwise plugin calls: UpdateState, then per cell a I - dS/dQ - dS/dAux
    dAux/dQ (a I below depth 1e-4), then per face in order the forward
    differences (eps 1e-7) of flux and fluctuations, scaled by area / volume,
    added into zeroed blocks.  The walls' boundary condition and the aux
    update do not depend on time or position for these plugins, so the
    pointwise calls (time 0, position 0) serve the boundary faces too."""
    m, model = c.mesh, c.model
    C, nq = x.shape
    xl = np.array([_pw(model, "update_variables", x[k], aux0[k], p) for k in range(C)])
    al = np.array([_pw(model, "update_aux_variables", xl[k], aux0[k], p) for k in range(C)])
    na = al.shape[1]
    D = np.zeros((C, nq, nq))
    for k in range(C):
        if nq > 1 and xl[k, 1] < 1e-4:
            J = np.zeros((nq, nq))
            J[np.arange(nq), np.arange(nq)] = a_shift
        else:
            dSdQ = _pw(model, "source_jacobian_wrt_variables", xl[k], al[k], p).reshape(nq, nq)
            dSdA = _pw(model, "source_jacobian_wrt_aux_variables", xl[k], al[k], p).reshape(nq, na)
            dAdQ = _pw(model, "aux_jacobian", xl[k], al[k], p).reshape(na, nq)
            J = np.empty((nq, nq))
            for i in range(nq):
                for j in range(nq):
                    dsrc = dSdQ[i, j]
                    for kk in range(na):
                        dsrc = dsrc + dSdA[i, kk] * dAdQ[kk, j]
                    J[i, j] = (a_shift if i == j else 0.0) - dsrc
        D[k] = 0.0 + J
    Po = np.zeros((m.n_faces, 2, nq, nq))
    eps = 1e-7
    fn = m.face_normal
    for f in range(m.n_faces):
        area = np.sqrt(sum(fn[f, d] * fn[f, d] for d in range(m.dim)))
        if area <= 1e-15:
            continue
        nh = np.zeros(3)
        nh[:m.dim] = fn[f, :m.dim] / area
        L, R = m.face_cells[f]
        fl = lambda qa, qb, aa, ab: _pw(model, "numerical_flux", qa, aa, p, n=nh, qR=qb, aR=ab)
        nc = lambda qa, qb, aa, ab: _pw(model, "numerical_fluctuations", qa, aa, p, n=nh, qR=qb, aR=ab)
        if R >= 0:
            Fb, NCb = fl(xl[L], xl[R], al[L], al[R]), nc(xl[L], xl[R], al[L], al[R])
            blocks = {}
            for side, (qs, as_) in enumerate(((xl[L], al[L]), (xl[R], al[R]))):
                J0, J1 = np.zeros((nq, nq)), np.zeros((nq, nq))
                for j in range(nq):
                    qp = qs.copy()
                    qp[j] += eps
                    ap = _pw(model, "update_aux_variables", qp, as_, p)
                    if side == 0:
                        Fp, NCp = fl(qp, xl[R], ap, al[R]), nc(qp, xl[R], ap, al[R])
                    else:
                        Fp, NCp = fl(xl[L], qp, al[L], ap), nc(xl[L], qp, al[L], ap)
                    dflux = (Fp - Fb) / eps
                    J0[:, j] = (0.0 + dflux) + (NCp[nq:] - NCb[nq:]) / eps
                    J1[:, j] = (0.0 - dflux) + (NCp[:nq] - NCb[:nq]) / eps
                blocks[side] = (J0, J1)
            fL, fR = area / m.cell_volume[L], area / m.cell_volume[R]
            JLL, JRL = blocks[0][0] * fL, blocks[0][1] * fR
            JLR, JRR = blocks[1][0] * fL, blocks[1][1] * fR
            D[L] = D[L] + JLL
            Po[f, 0] = 0.0 + JLR
            Po[f, 1] = 0.0 + JRL
            D[R] = D[R] + JRR
        elif m.face_bc[f] >= 0:
            assert m.face_bc[f] == 0
            qRb = _pw(model, "boundary_conditions", xl[L], al[L], p, n=nh)
            aRb = _pw(model, "update_aux_variables", qRb, al[L], p)
            Fb, NCb = fl(xl[L], qRb, al[L], aRb), nc(xl[L], qRb, al[L], aRb)
            J0 = np.zeros((nq, nq))
            for j in range(nq):
                qp = xl[L].copy()
                qp[j] += eps
                ap = _pw(model, "update_aux_variables", qp, al[L], p)
                qr = _pw(model, "boundary_conditions", qp, ap, p, n=nh)
                ar = _pw(model, "update_aux_variables", qr, ap, p)
                Fp, NCp = fl(qp, qr, ap, ar), nc(qp, qr, ap, ar)
                J0[:, j] = (0.0 + (Fp - Fb) / eps) + (NCp[nq:] - NCb[nq:]) / eps
            D[L] = D[L] + J0 * (area / m.cell_volume[L])
    return D, Po


@pytest.mark.parametrize("name", list(CASES))
def test_matrix_matches_plain_restatement(name):
    c = CASES[name]()
    o = _oracle(c)
    x = _perturbed(c)
    p = _params(c)
    a_shift = 437.5
    D, Po = o.implicit_jacobian(x, a_shift, t=0.0)
    Dr, Por = _restated_matrix(c, x, a_shift, p, o.get_aux())
    assert np.array_equal(D, Dr)
    assert np.array_equal(Po, Por)


def _dense(c, D, Po):
    C, nq = D.shape[0], D.shape[1]
    P = np.zeros((C * nq, C * nq))
    for k in range(C):
        P[k * nq:(k + 1) * nq, k * nq:(k + 1) * nq] = D[k]
    for f, (L, R) in enumerate(c.mesh.face_cells):
        if R >= 0:
            P[L * nq:(L + 1) * nq, R * nq:(R + 1) * nq] += Po[f, 0]
            P[R * nq:(R + 1) * nq, L * nq:(L + 1) * nq] += Po[f, 1]
    return P


@pytest.mark.parametrize("name", ["l2", "1d", "mixed"])
def test_matrix_is_the_jacobian_at_first_order(name):
    """At first order in space the faces see the cell states, so the
    assembled matrix is dF/dX (a = dXdot/dX): it agrees with central
    differences of the residual to their truncation error."""
    c = CASES[name]()
    o = _oracle(c, reconstruction_order=1)
    x = _perturbed(c)
    C, nq = x.shape
    a_shift = 250.0
    xn = x - 0.01
    F = lambda y: o.implicit_function(y, a_shift * (y - xn)).ravel()
    J = np.zeros((C * nq, C * nq))
    h = 1e-6
    xf = x.ravel()
    for j in range(C * nq):
        e = np.zeros_like(xf)
        e[j] = h
        J[:, j] = (F((xf + e).reshape(C, nq)) - F((xf - e).reshape(C, nq))) / (2 * h)
    P = _dense(c, *o.implicit_jacobian(x, a_shift))
    # the bathymetry columns are left out: far from the bump b is zero to
    # rounding in neighbouring cells, where the hydrostatic reconstruction's
    # max(b_L, b_R) has its kink and one-sided and central differences differ
    cols = np.arange(C * nq) % nq != 0
    scale = np.abs(J - a_shift * np.eye(C * nq)).max()
    assert np.abs(P - J)[:, cols].max() <= 1e-5 * scale


def _run(c, dts, **kw):
    o = _oracle(c, **kw)
    o.step(len(dts), dts=np.asarray(dts, dtype=float))
    return o


def test_bdf2_second_order_in_time():
    """First order in space, dt halved three times against a 64-step
    reference: BDF2 (order 1 on its first step) converges at second order."""
    O.set_threads(0)
    c = cases.level2(12)
    T = 0.01
    ref = _run(c, [T / 128] * 128, reconstruction_order=1).get_state()
    err = [np.linalg.norm(_run(c, [T / k] * k, reconstruction_order=1).get_state() - ref) for k in (8, 16, 32)]
    rates = np.log2(np.array(err[:-1]) / np.array(err[1:]))
    assert np.all((rates > 1.7) & (rates < 2.6)), (err, rates)


def test_lake_at_rest_and_mass():
    c = cases.level2(10)
    rest = dataclasses.replace(c)
    rest.q0 = c.q0.copy()
    rest.q0[:, 1] = 1.0 - rest.q0[:, 0]
    rest.q0[:, 2:] = 0.0
    o = _run(rest, [2e-3] * 5, reconstruction_order=1)
    q = o.get_state()
    assert np.abs(q[:, 0] + q[:, 1] - 1).max() < 1e-14 and np.abs(q[:, 2:]).max() < 1e-14
    assert o.implicit_stats()[0] == 0          # F(X_n) = 0: no Newton update needed
    for kw in ({"reconstruction_order": 1}, {"limiter": "none"}):
        o = _run(c, [1e-3] * 10, **kw)
        q = o.get_state()
        vol = c.mesh.cell_volume
        m0, m1 = (c.q0[:, 1] * vol).sum(), (q[:, 1] * vol).sum()
        assert abs(m1 - m0) < 1e-6 * m0, (kw, m1 - m0)
        assert o.implicit_stats()[3] > 0


def test_large_dt_with_stiff_source_stays_bounded():
    """Navier slip with slip length 1e-5 (friction rate about 1e4 per second)
    at ten times the explicit CFL step: BDF damps the moments."""
    c = cases.level2(10)
    names, _ = models.parameter_table(c.model)
    p = _params(c)
    p[names.index("lambda")] = 1e-5
    p[names.index("nu")] = 1e-1
    st = dataclasses.replace(c.settings, time_integration="implicit", reconstruction_order=1, cfl=4.5)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), st.to_struct(), p)
    o.set_state(c.q0)
    o.step(10)
    q = o.get_state()
    assert o.time()[0] > 0 and o.implicit_stats()[3] > 0
    assert np.all(np.isfinite(q)) and q[:, 1].min() > 0
    assert np.abs(q[:, 2:]).max() < np.abs(c.q0[:, 2:]).max()


def test_failed_newton_keeps_state_and_time():
    """With the TVD limiter at second order the residual is not differentiable
    at a state whose transverse moments are flat zero (any perturbation of one
    component switches the alpha all components share); GMRES on the
    difference quotients does not converge, the line search finds no descent,
    and the step is not taken."""
    c = cases.level2(4)
    o = _oracle(c)
    q0, (t0, _) = o.get_state(), o.time()
    o.step(1)
    assert o.implicit_stats()[3] == 0
    assert np.array_equal(o.get_state(), q0) and o.time()[0] == t0
