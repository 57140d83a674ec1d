"""The GPU discrete adjoint (zsme_adjoint) against the oracle.

* loss: the adjoint's forward run is the plain step, so its misfit equals
  the oracle's at the same dt sequence (the forward is bit-identical);
* directional derivatives: <grad, d> against the dual-number tangent-linear
  oracle run along d (the derivative of the same branches), for per-cell
  white-noise directions in the bathymetry b and for the Manning coefficient;
* central finite differences (eps = 1e-6) of the GPU forward with the
  recorded dts, on smooth directions over a horizon where the step is smooth
  on that scale;
* the torch.autograd wrapper returns the same gradients.
The case is the level-1 adjoint case (Manning friction, order 2, Green-Gauss,
Vacuum + TVD limiting) on small meshes; checkpoint intervals that do not
divide the step count exercise partial segments."""
import dataclasses

import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import adjoint as adj
from zoomy_dmplex_b200 import cases, models
from zoomy_dmplex_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals), names


def _smooth(mesh, rng, bumps=6):
    x, y = mesh.cell_centroid[:, 0], mesh.cell_centroid[:, 1]
    d = np.zeros_like(x)
    for _ in range(bumps):
        cx, cy = rng.uniform(0, 1, 2)
        w = rng.uniform(0.02, 0.1)
        d += rng.standard_normal() * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / w)
    return d


def _setup(n, nsteps, every_obs, ngauge, seed=0, mesh=None):
    c = cases.adjoint_l1(n, m=mesh)
    p, names = _params(c)
    tgt = cases.adjoint_l1(n, target=True, m=mesh)
    o = O.Oracle(tgt.model, tgt.mesh.as_abi_arrays(), tgt.settings.to_struct(), p)
    o.set_state(tgt.q0)
    steps = list(range(every_obs, nsteps + 1, every_obs))
    cells = adj.gauges(c.mesh.n_cells, ngauge, seed)
    targets = []
    for k in range(1, nsteps + 1):
        o.step(1)
        if k in steps:
            targets.append(o.get_state()[cells, 1])
    obs = adj.depth_observations(cells, steps, np.array(targets))
    return c, p, names, obs


def _oracle_tlm(c, p, dts, obs, dq, dp):
    """Misfit and its derivative along (dq, dp) from the tangent-linear oracle."""
    st, ce, co, tg = obs
    t = O.TangentOracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), p)
    t.set_state(c.q0)
    t.set_tangent(dq, dp)
    L = dL = 0.0
    for n in range(len(dts) + 1):
        sel = np.nonzero(st == n)[0]
        if sel.size:
            q, tan = t.get_state(), t.get_tangent()
            r = q[ce[sel], co[sel]] - tg[sel]
            L += float(np.sum(r * r))
            dL += float(np.sum(2.0 * r * tan[ce[sel], co[sel]]))
        if n < len(dts):
            t.step(1, dts=np.array([dts[n]]))
    return L, dL


@pytest.mark.parametrize("n,nsteps,every,mixed", [(16, 12, 5, False), (24, 30, 7, False), (14, 20, 6, True),
                                                  (16, 12, 4, False), (14, 20, 5, True)])
def test_adjoint_matches_tangent_linear_oracle(n, nsteps, every, mixed):
    """mixed: triangles and quadrilaterals in one mesh (empty face slots)."""
    from zoomy_dmplex_b200 import mesh as meshmod

    c, p, names, obs = _setup(n, nsteps, 3, 24, mesh=meshmod.mixed_square(n, seed=6) if mixed else None)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    loss, gq, gp, dts = g.adjoint(nsteps, *obs, checkpoint_every=every)
    # the handle ends at the state after nsteps plain steps
    h = Solver(c.model, c.mesh, c.settings, p)
    h.set_state(c.q0)
    h.step(nsteps)
    assert np.array_equal(g.get_state(), h.get_state())
    rng = np.random.default_rng(7)
    ni = names.index("n_manning")
    for what in ("b", "b", "manning"):
        dq = np.zeros_like(c.q0)
        dp = np.zeros_like(p)
        if what == "b":
            dq[:, 0] = rng.standard_normal(c.mesh.n_cells)
        else:
            dp[ni] = 1.0
        L, dL = _oracle_tlm(c, p, dts, obs, dq, dp)
        assert abs(L - loss) <= 1e-12 * abs(L)
        ad = float(np.sum(gq * dq) + np.sum(gp * dp))
        assert abs(ad - dL) <= 1e-8 * max(abs(dL), 1e-30), (what, ad, dL)


# separate face and gather kernels with the lean face-state kernel, and the
# fused tile kernel with the split face-state kernel
LAUNCHES = [None, {"prep": 64, "face": 128, "gather": 128, "finalize": 128, "prep_occ": 2, "face_occ": 4,
                   "finalize_occ": 3, "tile_faces": 128, "fuse_final": 0, "prep_lean": 2}]


@pytest.mark.parametrize("launch", LAUNCHES)
@pytest.mark.parametrize("nsteps,every", [(12, 4), (30, 5), (8, 4), (60, 3)])
def test_overlapped_replays_bitwise(nsteps, every, launch):
    """When every checkpoint segment is full, the replays run on a side
    stream into a second tape buffer while the reverse sweep runs; the loss,
    gradients, dts and final state equal those of the one-buffer form (forced
    by per-kernel timing, which runs plain launches) bit for bit, and the
    gradient agrees with the tangent-linear oracle."""
    from zoomy_dmplex_b200.solver import set_launch

    c, p, names, obs = _setup(20, nsteps, 2, 16)
    out = []
    for profiled in (False, True):
        g = Solver(c.model, c.mesh, c.settings, p)
        if launch:
            set_launch(g.h, launch)
        g.set_state(c.q0)
        g.set_profiling(profiled)
        r = g.adjoint(nsteps, *obs, checkpoint_every=every)
        assert g.adjoint_overlapped() == (not profiled)
        ph = g.adjoint_phases()
        assert min(ph.values()) >= 0.0
        out.append((r, g.get_state()))
        g.close()
    (l0, q0, p0, d0), s0 = out[0]
    (l1, q1, p1, d1), s1 = out[1]
    assert l0 == l1
    assert np.array_equal(q0, q1) and np.array_equal(p0, p1) and np.array_equal(d0, d1)
    assert np.array_equal(s0, s1)
    dq = np.zeros_like(c.q0)
    dq[:, 0] = np.random.default_rng(3).standard_normal(c.mesh.n_cells)
    L, dL = _oracle_tlm(c, p, d0, obs, dq, np.zeros_like(p))
    assert abs(L - l0) <= 1e-12 * abs(L)
    ad = float(np.sum(q0 * dq))
    assert abs(ad - dL) <= 1e-8 * max(abs(dL), 1e-30), (ad, dL)


def test_adjoint_matches_central_differences():
    n, nsteps = 16, 12
    c, p, names, obs = _setup(n, nsteps, 3, 24)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    loss, gq, gp, dts = g.adjoint(nsteps, *obs, checkpoint_every=5)
    st, ce, co, tg = obs

    def misfit(q0, pp):
        s = Solver(c.model, c.mesh, c.settings, pp)
        s.set_state(q0)
        L = 0.0
        for k in range(nsteps + 1):
            sel = np.nonzero(st == k)[0]
            if sel.size:
                r = s.get_state()[ce[sel], co[sel]] - tg[sel]
                L += float(np.sum(r * r))
            if k < nsteps:
                s.step(1, dts=dts[k:k + 1])
        return L

    assert abs(misfit(c.q0, p) - loss) <= 1e-13 * loss
    eps = 1e-6
    rng = np.random.default_rng(11)
    for _ in range(3):
        dq = np.zeros_like(c.q0)
        dq[:, 0] = _smooth(c.mesh, rng) * 1e-2
        fd = (misfit(c.q0 + eps * dq, p) - misfit(c.q0 - eps * dq, p)) / (2 * eps)
        ad = float(np.sum(gq * dq))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-14, (ad, fd)
    # The misfit's derivative in n is O(1e-7) here, and the Newton loop's
    # tolerance-based stop (0 or 1 update) moves the map in steps of up to its
    # 1e-8 tolerance, so central differences resolve it only to a few 1e-5
    # (2.7e-5 measured); the tangent-linear comparison above checks the same
    # derivative to 1e-8.
    dp = np.zeros_like(p)
    dp[names.index("n_manning")] = 1.0
    fd = (misfit(c.q0, p + eps * dp) - misfit(c.q0, p - eps * dp)) / (2 * eps)
    ad = float(np.sum(gp * dp))
    assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-14, (ad, fd)


def test_torch_autograd_wrapper():
    import torch

    n, nsteps = 16, 9
    c, p, names, obs = _setup(n, nsteps, 3, 16)
    g = Solver(c.model, c.mesh, c.settings, p)
    b = torch.tensor(c.q0[:, 0], requires_grad=True)
    pt = torch.tensor(p, requires_grad=True)
    rest = torch.tensor(c.q0[:, 1:])
    q0 = torch.cat([b[:, None], rest], dim=1)
    loss = adj.gauge_loss(g, q0, pt, nsteps, obs, checkpoint_every=4)
    (2.0 * loss).backward()
    g2 = Solver(c.model, c.mesh, c.settings, p)
    g2.set_state(c.q0)
    L, gq, gp, _ = g2.adjoint(nsteps, *obs, checkpoint_every=4)
    assert abs(float(loss.detach()) - L) <= 1e-14 * L
    assert np.allclose(b.grad.numpy(), 2.0 * gq[:, 0], rtol=0, atol=0)
    assert np.allclose(pt.grad.numpy(), 2.0 * gp, rtol=0, atol=0)


def test_adjoint_rejects_bad_input():
    from zoomy_dmplex_b200 import native

    c = cases.adjoint_l1(12)
    p, _ = _params(c)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    with pytest.raises(native.ZsmeError):
        g.adjoint(5, [9], [0], [1], [0.0])          # observation after the last step
    with pytest.raises(native.ZsmeError):
        g.adjoint(5, [1], [c.mesh.n_cells], [1], [0.0])


def test_dual_number_face_path_on_reference_style_header():
    """A plugin without a generated face VJP (the 1-D model mirrors the
    reference's shipped header) is differentiated by the dual-number face
    kernel: adjoint against the tangent-linear oracle."""
    from test_gpu_parity import case_1d

    c = case_1d()
    p, names = _params(c)
    nsteps = 20
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), p)
    q_tgt = c.q0.copy()
    q_tgt[:, 1] += 0.01 * np.exp(-(c.mesh.cell_centroid[:, 0] - 0.4) ** 2 / 0.02)
    o.set_state(q_tgt)
    steps = [5, 10, 15, 20]
    cells = adj.gauges(c.mesh.n_cells, 12, 3)
    targets = []
    for k in range(1, nsteps + 1):
        o.step(1)
        if k in steps:
            targets.append(o.get_state()[cells, 1])
    obs = adj.depth_observations(cells, steps, np.array(targets))
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    loss, gq, gp, dts = g.adjoint(nsteps, *obs, checkpoint_every=7)
    rng = np.random.default_rng(5)
    for _ in range(2):
        dq = np.zeros_like(c.q0)
        dq[:, 0] = rng.standard_normal(c.mesh.n_cells)
        L, dL = _oracle_tlm(c, p, dts, obs, dq, np.zeros_like(p))
        assert abs(L - loss) <= 1e-12 * abs(L)
        ad = float(np.sum(gq * dq))
        assert abs(ad - dL) <= 1e-8 * max(abs(dL), 1e-30), (ad, dL)


@pytest.mark.parametrize("kw", [{"reconstruction_order": 1}, {"ssp_stages": 3}, {"limiter": "none"}])
@pytest.mark.parametrize("every", [4, 5])
def test_adjoint_other_schemes(kw, every):
    """First order (one stage, no reconstruction record), three SSP stages (the
    reverse step's odd-stage path), no limiter; segments full (every 4: the
    overlapped replays) and partial (every 5): the directional derivatives
    agree with the tangent-linear oracle."""
    c, p, names, obs = _setup(16, 12, 3, 20)
    c.settings = dataclasses.replace(c.settings, **kw)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    loss, gq, gp, dts = g.adjoint(12, *obs, checkpoint_every=every)
    assert g.adjoint_overlapped() == (every == 4)
    rng = np.random.default_rng(11)
    ni = names.index("n_manning")
    for what in ("b", "manning"):
        dq = np.zeros_like(c.q0)
        dp = np.zeros_like(p)
        if what == "b":
            dq[:, 0] = rng.standard_normal(c.mesh.n_cells)
        else:
            dp[ni] = 1.0
        L, dL = _oracle_tlm(c, p, dts, obs, dq, dp)
        assert abs(L - loss) <= 1e-12 * abs(L), (kw, L, loss)
        ad = float(np.sum(gq * dq) + np.sum(gp * dp))
        assert abs(ad - dL) <= 1e-8 * max(abs(dL), 1e-30), (kw, what, ad, dL)
