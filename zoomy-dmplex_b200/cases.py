"""The benchmark cases: seeded synthetic meshes, initial conditions and
settings of the five configurations (SME level 0 plain, level 2, level 4 at
roofline size, the level-2 ensemble and the level-1 adjoint case).

The reference projects its initial condition onto cell centroids
(``VirtualSolver.hpp:258-281``); here the initial state is evaluated at the
centroids in numpy.  State layout: ``[b, h, hu_0..hu_L, hv_0..hv_L]``.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional

import numpy as np

from . import mesh as meshmod
from .settings import SolverSettings


def _gauss(x, y, cx, cy, w2):
    return np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / w2)


@dataclasses.dataclass
class Case:
    name: str
    model: str
    mesh: meshmod.Mesh
    q0: np.ndarray
    settings: SolverSettings
    params: Dict[str, float]
    steps: int


def _state(level, h, b, hu=None, hv=None):
    C = h.size
    nm = level + 1
    q = np.zeros((C, 2 + 2 * nm))
    q[:, 0] = b
    q[:, 1] = h
    if hu is not None:
        for k, v in enumerate(hu):
            q[:, 2 + k] = v
    if hv is not None:
        for k, v in enumerate(hv):
            q[:, 2 + nm + k] = v
    return q


def default_settings(**kw) -> SolverSettings:
    """Order 2 with Vacuum + TVD (Barth-Jespersen ratio) limiting, two-stage
    SSP-RK2, CFL 0.45, and the Green-Gauss gradient the reference's MUSCL path
    installs (``ModularSolver.hpp:62-67``).  The least-squares gradient
    (``gradient="least_squares"``) is never installed by that path; restated
    as written, its one-sided wall stencil lets wall cells grow without bound
    under inflow (flat bed, h = 1, u = 0.5 into reflective walls: |u| > 20 and
    h < 0 within 40 steps on an 80x80 grid, and the level-2 case below within
    100 steps), while Green-Gauss keeps the same runs bounded."""
    s = SolverSettings(t_end=1e9, cfl=0.45, reconstruction_order=2, limiter="tvd", ssp_stages=2,
                       gradient="green_gauss")
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def plain_l0(n: int = 60, seed: int = 0, steps: int = 200) -> Case:
    """SME level 0 (shallow water), hump over a Gaussian bump, Manning n=0.03,
    with the least-squares gradient and Barth-Jespersen (Vacuum + TVD)
    limiting the configuration names.  The flow starts at rest and stays
    bounded over its 200 steps with the one-sided least-squares wall stencil
    (oracle, 60x60 grid: depth within [0.80, 1.05], |u| <= 0.25), unlike the
    inflow cases of default_settings."""
    m = meshmod.jittered_square(n, seed=seed)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = 0.2 * _gauss(x, y, 0.5, 0.5, 0.01)
    h = 1.0 - b + 0.05 * _gauss(x, y, 0.3, 0.3, 0.005)
    q = _state(0, h, b)
    return Case("plain_l0_%d" % n, "sme2d_l0", m, q, default_settings(gradient="least_squares"),
                dict(g=9.81, n_manning=0.03, nu=0.0), steps)


def level2(n: int = 240, seed: int = 1, steps: int = 500) -> Case:
    """SME level 2: same bathymetry and hump, u = 0.5, alpha_1 = 0.1,
    Navier slip lambda = 0.1, nu = 1e-3."""
    m = meshmod.jittered_square(n, seed=seed)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = 0.2 * _gauss(x, y, 0.5, 0.5, 0.01)
    h = 1.0 - b + 0.05 * _gauss(x, y, 0.3, 0.3, 0.005)
    q = _state(2, h, b, hu=[0.5 * h, 0.1 * h, 0 * h], hv=[0 * h] * 3)
    return Case("level2_%d" % n, "sme2d_l2", m, q, default_settings(),
                dict(g=9.81, nu=1e-3, **{"lambda": 0.1}, n_manning=0.0), steps)


def mixed_level2(n: int = 24, seed: int = 5, steps: int = 60) -> Case:
    """The level-2 problem (bathymetry, hump, u = 0.5, alpha_1 = 0.1, Navier
    slip) on a mesh of mixed triangles and quadrilaterals (mesh.mixed_square:
    -1 padded cells, so triangles have an empty face slot)."""
    m = meshmod.mixed_square(n, seed=seed)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = 0.2 * _gauss(x, y, 0.5, 0.5, 0.01)
    h = 1.0 - b + 0.05 * _gauss(x, y, 0.3, 0.3, 0.005)
    q = _state(2, h, b, hu=[0.5 * h, 0.1 * h, 0 * h], hv=[0 * h] * 3)
    return Case("mixed_level2_%d" % n, "sme2d_l2", m, q, default_settings(),
                dict(g=9.81, nu=1e-3, **{"lambda": 0.1}, n_manning=0.0), steps)


def roofline_l4(n: int = 1400, seed: int = 2, steps: int = 100, m: Optional[meshmod.Mesh] = None) -> Case:
    """SME level 4 at roofline size: bathymetry = 16 seeded Gaussians
    (amplitude U[0.02,0.1], width U[0.02,0.08], centre U[0,1]^2),
    h = 1 - b + U(+-0.01), alpha_1 ~ U[0, 0.05], other moments 0."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.02, 0.1, 16)
    wid = rng.uniform(0.02, 0.08, 16)
    cen = rng.uniform(0.0, 1.0, (16, 2))
    if m is None:
        m = meshmod.jittered_square(n, seed=seed)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = np.zeros_like(x)
    for a, w, c in zip(amp, wid, cen):
        b += a * _gauss(x, y, c[0], c[1], w * w)
    h = 1.0 - b + rng.uniform(-0.01, 0.01, x.size)
    a1 = rng.uniform(0.0, 0.05, x.size)
    q = _state(4, h, b, hu=[0 * h, a1 * h] + [0 * h] * 3, hv=[0 * h] * 5)
    return Case("roofline_l4_%d" % n, "sme2d_l4", m, q, default_settings(),
                dict(g=9.81, nu=1e-3, **{"lambda": 0.1}, n_manning=0.0), steps)


def wet_dry_patchwork(n: int = 24, seed: int = 12, level: int = 0) -> Case:
    """Wet/dry patchwork for the positivity variants: each cell dry with
    probability 1/2, else depth U[0.01, 0.3] with velocities U[-3, 3]^2, over
    three Gaussian bumps (amplitude U[0, 0.2], width^2 U[0.005, 0.03]); no
    friction.  At CFL 1.5 the limited order-2 step drives depths negative
    within the first steps, which the MOOD variant repairs."""
    rng = np.random.default_rng(seed)
    m = meshmod.jittered_square(n, seed=7)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = np.zeros_like(x)
    for _ in range(3):
        a = rng.uniform(0, 0.2)
        c = rng.uniform(0, 1, 2)
        b = b + a * _gauss(x, y, c[0], c[1], rng.uniform(0.005, 0.03))
    h = np.where(rng.uniform(0, 1, x.size) < 0.5, 0.0, rng.uniform(0.01, 0.3, x.size))
    u = rng.uniform(-3, 3, x.size)
    v = rng.uniform(-3, 3, x.size)
    q = _state(level, h, b, hu=[h * u] + [0 * h] * level, hv=[h * v] + [0 * h] * level)
    return Case("wet_dry_patchwork_%d" % n, "sme2d_l%d" % level, m, q, default_settings(cfl=1.5),
                dict(g=9.81, nu=0.0, n_manning=0.0), 20)


def ensemble_side(i: int, seed: int = 3, side_range=(40, 400)) -> int:
    """Grid side of ensemble instance i (the first draw of its generator)."""
    rng = np.random.default_rng([seed, i])
    return int(round(np.exp(rng.uniform(np.log(side_range[0]), np.log(side_range[1])))))


def shard_instances(cells, world: int):
    """Instances over `world` ranks by greedy balance on their cell counts
    (largest first, each to the least loaded rank; ties to the lower rank):
    list of index lists, each in increasing order."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += cells[i]
        out[r].append(i)
    return [sorted(o) for o in out]


def ensemble_shard(n_total: int, world: int, rank: int, seed: int = 3, side_range=(40, 400)):
    """The instance indices rank `rank` of `world` advances: greedy balance
    on the cell counts 2 (side - 1)^2 of the Delaunay grids."""
    cells = [2 * (ensemble_side(i, seed, side_range) - 1) ** 2 for i in range(n_total)]
    return shard_instances(cells, world)[rank]


def ensemble_member(i: int, seed: int = 3, side_range=(40, 400)) -> Case:
    """Instance i of the level-2 ensemble: grid side log-uniform in
    [40, 400], 1-4 Gaussian bumps (amplitude U[0.05,0.2], width
    U[0.005,0.03]), one hump (amplitude U[0.01,0.1])."""
    rng = np.random.default_rng([seed, i])
    side = int(round(np.exp(rng.uniform(np.log(side_range[0]), np.log(side_range[1])))))
    m = meshmod.jittered_square(side, seed=int(rng.integers(1 << 30)))
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = np.zeros_like(x)
    for _ in range(int(rng.integers(1, 5))):
        a, w2 = rng.uniform(0.05, 0.2), rng.uniform(0.005, 0.03)
        c = rng.uniform(0.2, 0.8, 2)
        b += a * _gauss(x, y, c[0], c[1], w2)
    c = rng.uniform(0.2, 0.8, 2)
    h = 1.0 - b + rng.uniform(0.01, 0.1) * _gauss(x, y, c[0], c[1], 0.005)
    q = _state(2, h, b, hu=[0 * h] * 3, hv=[0 * h] * 3)
    return Case("ensemble_%d" % i, "sme2d_l2", m, q, default_settings(),
                dict(g=9.81, nu=1e-3, **{"lambda": 0.1}, n_manning=0.0), 200)


def adjoint_l1(n: int = 200, seed: int = 4, steps: int = 400, target: bool = False,
               m: Optional[meshmod.Mesh] = None) -> Case:
    """SME level 1 adjoint case, Manning n = 0.03; the target run perturbs b by
    +0.02 exp(-((x-0.6)^2+(y-0.4)^2)/0.01).

    The state is chosen so that the discrete step is differentiable where it
    starts: b = 0.2 bump + a bowl 0.1 |x - (0.4, 0.55)|^2, so that no
    component is flat to round-off (a TVD ratio with |dq| just above the
    reference's 1e-12 cut-off has an arbitrarily large slope); every velocity
    and moment is non-zero (|u| at u = 0 is a kink of the Rusanov speed), with
    the flow tapered towards the reflective walls.  m: another mesh of the
    unit square (default: the jittered n x n triangulation)."""
    if m is None:
        m = meshmod.jittered_square(n, seed=seed)
    x, y = m.cell_centroid[:, 0], m.cell_centroid[:, 1]
    b = 0.2 * _gauss(x, y, 0.5, 0.5, 0.01) + 0.1 * ((x - 0.4) ** 2 + (y - 0.55) ** 2)
    if target:
        b = b + 0.02 * _gauss(x, y, 0.6, 0.4, 0.01)
    h = 1.0 - b + 0.05 * _gauss(x, y, 0.3, 0.3, 0.005) + 0.02 * x
    w = (np.sin(np.pi * x) * np.sin(np.pi * y)) ** 2
    u0 = w * (0.3 + 0.05 * np.sin(2 * np.pi * y)) + 0.02
    v0 = w * (0.15 + 0.05 * np.cos(2 * np.pi * x)) + 0.01
    q = _state(1, h, b, hu=[h * u0, h * 0.05 * w * (1 + 0.3 * x)],
               hv=[h * v0, -h * 0.03 * w * (1 + 0.2 * y)])
    return Case("adjoint_l1_%d" % n, "sme2d_l1", m, q, default_settings(),
                dict(g=9.81, n_manning=0.03, nu=0.0), steps)


def _member(args):
    i, seed, lo, hi = args
    return ensemble_member(i, seed=seed, side_range=(lo, hi))


def ensemble(n: int = 512, seed: int = 3, side_range=(40, 400), processes: int = 0, first: int = 0,
             indices=None):
    """Instances first .. first+n-1 (or the given indices) of the level-2
    ensemble, built in parallel worker processes (spawned, so it is safe
    after CUDA has been initialised)."""
    import multiprocessing as mp
    import os

    idx = list(indices) if indices is not None else list(range(first, first + n))
    n = len(idx)
    args = [(i, seed, side_range[0], side_range[1]) for i in idx]
    procs = processes or min(n, os.cpu_count() or 1)
    if procs <= 1 or n < 4:
        return [_member(a) for a in args]
    with mp.get_context("spawn").Pool(procs) as pool:
        return pool.map(_member, args, chunksize=1)
