"""The solver subset of the reference's JSON settings.

Mirrors ``Settings::from_json`` (reference ``Settings.hpp:73-138``) for the
keys that change the SME step, with the same defaults, plus the model
parameter overrides by name (``VirtualSolver.hpp:199-217``).  Two keys are
additions of this implementation: ``solver.gradient`` (``"green_gauss"``, the
default and the gradient the reference's MUSCL path installs,
``ModularSolver.hpp:62-67``, or ``"least_squares"``, the reference's
``LeastSquaresGradient`` of ``Gradient.hpp:196-360``, which its MUSCL path
never installs; its one-sided stencil at reflective walls lets wall cells
grow without bound under inflow, so it is an option, not the default) and
``solver.block_size``.

How the reference interprets the strings, and so how they map here:
* ``limiter``: only ``"none"`` changes anything; every other value (including
  the default ``"venkatakrishnan"``) installs Vacuum + TVD limiting through
  the backward-compatible ``LinearReconstructor`` constructor
  (``MUSCLSolver.hpp:43``, ``Reconstruction.hpp:170-175``);
* ``time_integration``: ``"splitting"`` (explicit transport, then the implicit
  source step) or ``"imex"`` (the additive Runge-Kutta scheme 2E of the
  reference's IMEX strategy, explicit transport and implicit source in every
  stage, at the step's CFL dt) or ``"implicit"`` (the fully implicit strategy:
  BDF2 of the transport and the source together, Newton with a matrix-free
  Jacobian and GMRES preconditioned by the diagonal blocks of the reference's
  assembled Jacobian, at the step's CFL dt; single meshes, positivity other
  than ``"mood"``);
* ``refresh_derivative_aux`` (reference default true): before each state
  update the plugin's derivative aux slots are refilled with Green-Gauss
  derivatives of the state (``TransportStep.hpp:161-202``); plugins without
  the field-level ``update_aux_variables`` overload have nothing to refresh;
* ``positivity``: ``"none"`` (limited linear reconstruction), ``"zhang_shu"``
  or ``"mood"`` (the eta-well-balanced reconstruction with the Zhang-Shu
  theta, or with the a-posteriori first-order override of cells that end
  with negative depth), with ``wet_dry_eps`` the dry threshold.
"""
from __future__ import annotations

import dataclasses
import json
from typing import Dict, Optional

from . import native


@dataclasses.dataclass
class SolverSettings:
    t_end: float = 1.0
    cfl: float = 0.5
    reconstruction_order: int = 1
    min_dt: float = 1.0e-12
    limiter: str = "venkatakrishnan"
    time_integration: str = "splitting"
    positivity: str = "none"
    wet_dry_eps: float = 1.0e-2
    ssp_stages: int = 5
    gradient: str = "green_gauss"
    block_size: int = 0
    refresh_derivative_aux: bool = True

    def to_struct(self) -> native.ZsmeSettings:
        if self.time_integration not in native.TIME_INTEGRATION:
            raise ValueError("time_integration must be 'splitting', 'imex' or 'implicit', not %r"
                             % self.time_integration)
        if self.positivity not in native.POSITIVITY:
            raise ValueError("positivity must be one of %s" % sorted(native.POSITIVITY))
        if self.gradient not in ("least_squares", "green_gauss"):
            raise ValueError("gradient must be 'least_squares' or 'green_gauss'")
        if self.reconstruction_order >= 2 and self.ssp_stages < 2:
            raise ValueError("ssp_stages must be >= 2")
        s = native.ZsmeSettings()
        s.cfl, s.t_end, s.min_dt = self.cfl, self.t_end, self.min_dt
        s.reconstruction_order = int(self.reconstruction_order)
        s.limiter = native.ZSME_LIMITER_NONE if self.limiter == "none" else native.ZSME_LIMITER_TVD
        s.gradient = (native.ZSME_GRADIENT_LSQ if self.gradient == "least_squares"
                      else native.ZSME_GRADIENT_GREEN_GAUSS)
        s.ssp_stages = int(self.ssp_stages)
        s.source = 1
        s.block_size = int(self.block_size)
        s.positivity = native.POSITIVITY[self.positivity]
        s.wet_dry_eps = float(self.wet_dry_eps)
        s.refresh_derivative_aux = 1 if self.refresh_derivative_aux else 0
        s.time_integration = native.TIME_INTEGRATION[self.time_integration]
        return s


@dataclasses.dataclass
class Settings:
    name: str = "Simulation"
    solver: SolverSettings = dataclasses.field(default_factory=SolverSettings)
    parameters: Dict[str, float] = dataclasses.field(default_factory=dict)

    @staticmethod
    def from_dict(j: dict) -> "Settings":
        s = Settings(name=j.get("name", "Simulation"))
        js = j.get("solver", {})
        d = SolverSettings()
        for f in dataclasses.fields(SolverSettings):
            if f.name in js:
                setattr(d, f.name, type(getattr(d, f.name))(js[f.name]))
        s.solver = d
        for k, v in j.get("model", {}).get("parameters", {}).items():
            if isinstance(v, (int, float)):
                s.parameters[k] = float(v)
        return s

    @staticmethod
    def from_json(path: str) -> "Settings":
        with open(path) as f:
            return Settings.from_dict(json.load(f))


def resolve_parameters(names, defaults, overrides: Optional[Dict[str, float]]):
    """Model parameter vector with overrides by name; unknown names are
    reported and ignored, as the reference does."""
    p = [float(v) for v in defaults]
    unknown = []
    for k, v in (overrides or {}).items():
        if k in names:
            p[names.index(k)] = float(v)
        else:
            unknown.append(k)
    return p, unknown
