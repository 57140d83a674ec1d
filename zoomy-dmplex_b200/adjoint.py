"""Gradients of an SME run through its discrete adjoint, as a torch op.

``gauge_loss(solver, q0, params, nsteps, obs)`` runs ``nsteps`` steps of
``solver`` from the state ``q0`` ([n_cells, n_dof_q], caller cell order) with
the model parameters ``params`` and returns the least-squares misfit at the
observations ``obs = (step, cell, comp, target[, weight])``:

    loss = sum_j w_j (Q_{step_j}[cell_j, comp_j] - target_j)^2 .

The forward call already runs the adjoint (``zsme_adjoint``: checkpoints
every ``checkpoint_every`` steps, recomputation in between) and keeps the
gradients; ``backward`` scales them by the incoming gradient.  Column 0 of
the state gradient is the gradient with respect to the bathymetry b, so a
caller that builds ``q0`` from a bathymetry tensor by torch operations gets
d loss / d b by ordinary autograd.  The CFL dt of every step is the one of
the forward run and is held fixed by the derivative (it is returned in
``GaugeLoss.last_dts``).
"""
from __future__ import annotations

import numpy as np
import torch


class GaugeLoss(torch.autograd.Function):
    last_dts = None

    @staticmethod
    def forward(ctx, q0, params, solver, nsteps, obs, checkpoint_every):
        solver.set_params(params.detach().to("cpu", torch.float64).numpy())
        solver.set_state(q0.detach().to("cpu", torch.float64).numpy())
        weight = obs[4] if len(obs) > 4 else None
        loss, gq, gp, dts = solver.adjoint(nsteps, obs[0], obs[1], obs[2], obs[3], weight,
                                           checkpoint_every=checkpoint_every)
        GaugeLoss.last_dts = dts
        ctx.save_for_backward(torch.from_numpy(gq).to(q0.device, q0.dtype),
                              torch.from_numpy(gp).to(params.device, params.dtype))
        return torch.tensor(loss, dtype=q0.dtype, device=q0.device)

    @staticmethod
    def backward(ctx, g):
        gq, gp = ctx.saved_tensors
        return g * gq, g * gp, None, None, None, None


def gauge_loss(solver, q0: torch.Tensor, params: torch.Tensor, nsteps: int, obs, checkpoint_every: int = 20):
    """The misfit as a differentiable function of ``q0`` and ``params``."""
    return GaugeLoss.apply(q0, params, solver, int(nsteps), obs, int(checkpoint_every))


def gauges(n_cells: int, n: int = 64, seed: int = 0) -> np.ndarray:
    """n distinct seeded gauge cells."""
    return np.random.default_rng(seed).choice(n_cells, size=n, replace=False).astype(np.int32)


def depth_observations(cells, steps, targets):
    """Observations of the depth (component 1) at ``cells`` after each of
    ``steps``; ``targets[k, g]`` is the target at steps[k], cells[g]."""
    cells = np.asarray(cells, dtype=np.int32)
    steps = np.asarray(steps, dtype=np.int32)
    st = np.repeat(steps, cells.size)
    ce = np.tile(cells, steps.size)
    co = np.ones_like(ce)
    return st, ce, co, np.asarray(targets, dtype=np.float64).reshape(-1)


def observe_run(solver, q0, nsteps: int, steps, cells, comp: int = 1, dts=None) -> np.ndarray:
    """Values of component ``comp`` at ``cells`` after each of ``steps`` in a
    plain run of ``solver`` from ``q0`` (CFL dts, or the given ``dts``):
    targets for ``depth_observations``, or the misfit of a perturbed run."""
    steps = sorted(int(s) for s in steps)
    cells = np.asarray(cells)
    solver.set_state(q0)
    out = []
    k = 0
    for s in steps:
        if s > k:
            solver.step(s - k, None if dts is None else dts[k:s])
            k = s
        out.append(solver.get_state()[cells, comp])
    return np.array(out)


def smooth_direction(mesh, rng, bumps: int = 6) -> np.ndarray:
    """A seeded random smooth per-cell field (a sum of Gaussians with random
    centres, widths and signs): a direction along which the discrete step is
    smooth on the scale of a finite-difference check."""
    x, y = mesh.cell_centroid[:, 0], mesh.cell_centroid[:, 1]
    d = np.zeros_like(x)
    for _ in range(bumps):
        cx, cy = rng.uniform(0, 1, 2)
        w = rng.uniform(0.02, 0.1)
        d += rng.standard_normal() * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / w)
    return d
