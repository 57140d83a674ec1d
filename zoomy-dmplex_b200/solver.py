"""Host driver over the C ABI, shaped like the reference's MUSCLSolver.

``Solver`` owns one ``zsme_handle``: the mesh and the model live on the GPU
from construction on; ``set_state`` loads an initial condition (caller cell
order, ``[n_cells, n_dof_q]``), ``step`` advances whole time steps on the
device (one CUDA graph per step, no host synchronisation), ``run`` mirrors
``MUSCLSolver::Run``'s ``while (time < t_end)`` loop (reference
``MUSCLSolver.hpp:140-188``).  The individual hot-path calls are exposed
too: ``rhs`` (``TransportStep::FormRHS``), ``update_state``
(``TransportStep::UpdateState``), ``source`` (``SourceStep::Solve``) and
``compute_dt`` (``VirtualSolver::ComputeTimeStep``).
"""
from __future__ import annotations

import ctypes as ct
from typing import Dict, Optional, Union

import numpy as np

from . import native
from .mesh import Mesh
from .settings import Settings, SolverSettings, resolve_parameters


def _p(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


class Solver:
    def __init__(self, model: str, mesh: Mesh, settings: Union[Settings, SolverSettings, None] = None,
                 params: Union[None, Dict[str, float], np.ndarray, list] = None, device: int = 0):
        self.lib = native.load()
        self.model = model
        self.info = native.model_info(model)
        self.nq = self.info["n_dof_q"]
        self.naux = self.info["n_dof_qaux"]
        if isinstance(settings, Settings):
            overrides = dict(settings.parameters)
            solver_settings = settings.solver
        else:
            overrides = {}
            solver_settings = settings or SolverSettings()
        self.settings = solver_settings
        self.params = self._resolve_params(params, overrides)
        self.mesh = mesh
        self.C = mesh.n_cells
        self._mesh_keep = native.make_mesh_struct(mesh.as_abi_arrays())
        self._st = solver_settings.to_struct()
        h = ct.c_void_p()
        native.check(self.lib.zsme_create(model.encode(), ct.addressof(self._mesh_keep[0]),
                                          ct.addressof(self._st), _p(self.params), int(device), ct.byref(h)))
        self.h = h

    def _resolve_params(self, params, overrides):
        from . import models as _m
        names, defaults = _m.parameter_table(self.model)
        if params is None or isinstance(params, dict):
            merged = dict(overrides)
            merged.update(params or {})
            vals, unknown = resolve_parameters(names, defaults, merged)
            if unknown:
                raise KeyError("parameters not defined by model %s: %s" % (self.model, unknown))
            return np.ascontiguousarray(vals, dtype=np.float64)
        a = np.ascontiguousarray(params, dtype=np.float64)
        if a.size != len(names):
            raise ValueError("expected %d parameters" % len(names))
        return a

    def close(self):
        if getattr(self, "h", None):
            self.lib.zsme_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ state
    def set_state(self, q: np.ndarray, t: float = 0.0):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.C, self.nq)
        native.check(self.lib.zsme_set_state(self.h, _p(q), float(t)))

    def set_state_device(self, q_dev_ptr: int, t: float = 0.0):
        native.check(self.lib.zsme_set_state_device(self.h, ct.c_void_p(q_dev_ptr), float(t)))

    def get_state(self) -> np.ndarray:
        q = np.empty((self.C, self.nq))
        native.check(self.lib.zsme_get_state(self.h, _p(q)))
        return q

    def get_state_device(self, q_dev_ptr: int):
        native.check(self.lib.zsme_get_state_device(self.h, ct.c_void_p(q_dev_ptr)))

    def get_cells(self, cells) -> np.ndarray:
        """zsme_get_cells: the state of the given cells (caller ids), [n, nq]."""
        c = np.ascontiguousarray(cells, dtype=np.int32)
        q = np.empty((len(c), self.nq))
        native.check(self.lib.zsme_get_cells(self.h, len(c), c.ctypes.data_as(ct.c_void_p), _p(q), 0))
        return q

    def set_cells(self, cells, q):
        """zsme_set_cells: the state of the given cells (caller ids) and their
        aux variables; time and dt unchanged."""
        c = np.ascontiguousarray(cells, dtype=np.int32)
        q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).reshape(len(c), self.nq))
        native.check(self.lib.zsme_set_cells(self.h, len(c), c.ctypes.data_as(ct.c_void_p), _p(q), 0))

    def set_state_async(self, q_host_ptr: int, t: float = 0.0):
        """zsme_set_state_async: the state at host address q_host_ptr (AoS,
        caller order; page-locked for a truly asynchronous copy) becomes the
        state at time t once the handle's stream reaches it.  The buffer must
        stay unchanged until sync()."""
        native.check(self.lib.zsme_set_state_async(self.h, ct.c_void_p(q_host_ptr), float(t)))

    def get_state_async(self, q_host_ptr: int):
        """zsme_get_state_async: the current state is copied to host address
        q_host_ptr; valid after sync()."""
        native.check(self.lib.zsme_get_state_async(self.h, ct.c_void_p(q_host_ptr)))

    def stream_wait_copies(self):
        """The handle's stream waits (on the device) for the asynchronous copies issued so far."""
        native.check(self.lib.zsme_stream_wait_copies(self.h))

    def get_aux(self) -> np.ndarray:
        a = np.empty((self.C, self.naux))
        native.check(self.lib.zsme_get_aux(self.h, _p(a)))
        return a

    def set_params(self, params):
        self.params = np.ascontiguousarray(params, dtype=np.float64)
        native.check(self.lib.zsme_set_params(self.h, _p(self.params)))

    # ------------------------------------------------------- hot-path calls
    def rhs(self, x: np.ndarray, t: float = 0.0) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        f = np.empty_like(x)
        native.check(self.lib.zsme_rhs(self.h, float(t), _p(x), _p(f)))
        return f

    def implicit_function(self, x: np.ndarray, xdot: np.ndarray, t: float = 0.0) -> np.ndarray:
        """F(t, X, Xdot) = Xdot - S(X) - R(X) of the fully implicit strategy
        (IFunctionWrapper, SolverStrategies.hpp:163-174)."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        xd = np.ascontiguousarray(xdot, dtype=np.float64).reshape(self.C, self.nq)
        f = np.empty_like(x)
        native.check(self.lib.zsme_implicit_function(self.h, float(t), _p(x), _p(xd), _p(f)))
        return f

    def implicit_jacobian(self, x: np.ndarray, shift: float, t: float = 0.0):
        """The implicit strategy's assembled matrix at (t, X, shift)
        (FormImplicitJacobian, ModularSolver.hpp:238-371): diagonal blocks
        [C, nq, nq] and per face the (L, R) and (R, L) blocks [F, 2, nq, nq]."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        d = np.empty((self.C, self.nq, self.nq))
        o = np.empty((self.mesh.n_faces, 2, self.nq, self.nq))
        native.check(self.lib.zsme_implicit_jacobian(self.h, float(t), _p(x), float(shift), _p(d), _p(o)))
        return d, o

    def implicit_stats(self):
        """Last implicit step: Newton iterations, GMRES iterations, line-search
        halvings, stop reason (1 residual, 2 update size, 0 neither)."""
        v = (ct.c_int32 * 4)()
        native.check(self.lib.zsme_implicit_stats(self.h, v))
        return [int(x) for x in v]

    def update_state(self):
        native.check(self.lib.zsme_update_state(self.h))

    def source(self, dt: float):
        native.check(self.lib.zsme_source(self.h, float(dt)))

    def compute_dt(self) -> float:
        d = ct.c_double()
        native.check(self.lib.zsme_compute_dt(self.h, ct.byref(d)))
        return d.value

    def step(self, n: int = 1, dts: Optional[np.ndarray] = None):
        if dts is None:
            native.check(self.lib.zsme_step(self.h, int(n)))
        else:
            d = np.ascontiguousarray(dts, dtype=np.float64)
            native.check(self.lib.zsme_step_dt(self.h, int(d.size), _p(d)))

    def sync(self, check: bool = True) -> native.ZsmeDiag:
        d = native.ZsmeDiag()
        native.check(self.lib.zsme_get_diag(self.h, ct.byref(d)))
        if check:
            native.check(self.lib.zsme_sync(self.h))
        return d

    def adjoint(self, nsteps: int, obs_step, obs_cell, obs_comp, obs_target, obs_weight=None,
                checkpoint_every: int = 20):
        """Discrete adjoint of ``nsteps`` steps from the current state.

        Loss = sum_j w_j (Q_{obs_step[j]}[obs_cell[j], obs_comp[j]] - obs_target[j])^2
        with Q_k the state after k steps (caller cell order).  Returns
        ``(loss, grad_q [n_cells, n_dof_q], grad_params [n_parameters], dts
        [nsteps])``: the gradients with respect to the current state (column 0
        is the bathymetry) and the parameters, at the dt sequence of the
        forward run (``dts``), which the derivative holds fixed.  Afterwards
        the solver holds the state after ``nsteps`` steps.  Checkpoints every
        ``checkpoint_every`` steps; the reverse pass recomputes in between."""
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        st, ce, co, tg = i32(obs_step), i32(obs_cell), i32(obs_comp), f64(obs_target)
        n = st.size
        if not (ce.size == co.size == tg.size == n):
            raise ValueError("observation arrays differ in length")
        wt = None if obs_weight is None else f64(obs_weight)
        if wt is not None and wt.size != n:
            raise ValueError("observation weights differ in length")
        ip = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_int32))
        loss = np.zeros(1)
        gq = np.zeros((self.mesh.n_cells, self.nq))
        gp = np.zeros(self.info["n_parameters"])
        dts = np.zeros(max(1, int(nsteps)))
        native.check(self.lib.zsme_adjoint(self.h, int(nsteps), int(checkpoint_every), n, ip(st), ip(ce), ip(co),
                                           _p(tg), _p(wt) if wt is not None else None, _p(loss), _p(gq), _p(gp),
                                           _p(dts)))
        return float(loss[0]), gq, gp, dts[:int(nsteps)]

    def adjoint_phases(self):
        """Device ms of the last adjoint call: forward pass, replays, reverse sweep."""
        ms = np.zeros(3)
        native.check(self.lib.zsme_adjoint_phases(self.h, _p(ms)))
        return {"forward": float(ms[0]), "replay": float(ms[1]), "reverse": float(ms[2])}

    def adjoint_overlapped(self):
        """Whether the last adjoint call overlapped its segment replays with
        the reverse sweep; then "replay" in adjoint_phases() is the first
        replay alone and "reverse" the rest of the reverse phase."""
        v = ct.c_int32()
        native.check(self.lib.zsme_adjoint_overlapped(self.h, ct.byref(v)))
        return bool(v.value)

    def time(self):
        t, d = ct.c_double(), ct.c_double()
        native.check(self.lib.zsme_get_time(self.h, ct.byref(t), ct.byref(d)))
        return t.value, d.value

    def run(self, max_steps: int = 1 << 30, chunk: int = 50):
        """MUSCLSolver::Run's loop: step until t >= t_end (checked every
        `chunk` steps; steps past t_end are no-ops on the device)."""
        done = 0
        while done < max_steps:
            n = min(chunk, max_steps - done)
            self.step(n)
            done += n
            t, _ = self.time()
            if t >= self.settings.t_end:
                break
        return self.sync()

    @property
    def stream(self) -> int:
        return self.lib.zsme_stream(self.h) or 0

    def set_profiling(self, on: bool = True):
        native.check(self.lib.zsme_set_profiling(self.h, int(bool(on))))

    def read_profile(self):
        """{kernel kind: (summed ms, launches)} since set_profiling(True)."""
        k = len(native.KERNEL_KINDS)
        ms = np.zeros(k)
        n = (ct.c_int64 * k)()
        native.check(self.lib.zsme_read_profile(self.h, _p(ms), n))
        return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(native.KERNEL_KINDS)}

    def launches_per_step(self) -> int:
        n = ct.c_int32()
        native.check(self.lib.zsme_launches_per_step(self.h, ct.byref(n)))
        return n.value


class BatchSolver:
    """An ensemble of independent instances (own mesh, parameters, time and
    CFL dt) advanced together: every kernel launch of ``step`` covers all
    instances (concatenated cell and face layout)."""

    def __init__(self, model: str, meshes, settings: Union[SolverSettings, None] = None, params=None,
                 device: int = 0):
        from . import models as _m
        self.lib = native.load()
        self.model = model
        self.info = native.model_info(model)
        self.nq = self.info["n_dof_q"]
        self.settings = settings or SolverSettings()
        self.meshes = list(meshes)
        self.n = len(self.meshes)
        # instances with fewer face slots (triangles beside quadrilaterals)
        # get empty slots, so every instance has the same max_faces
        kmax = max(m.max_faces for m in self.meshes)
        if any(m.max_faces != kmax for m in self.meshes):
            from .mesh import pad_face_slots
            self.meshes = [pad_face_slots(m, kmax) for m in self.meshes]
        names, defaults = _m.parameter_table(model)
        P = np.zeros((self.n, len(names)))
        for i in range(self.n):
            pi = params[i] if isinstance(params, (list, tuple)) else params
            if pi is None or isinstance(pi, dict):
                vals, unknown = resolve_parameters(names, defaults, pi or {})
                if unknown:
                    raise KeyError("parameters not defined by model %s: %s" % (model, unknown))
                P[i] = vals
            else:
                P[i] = np.asarray(pi, dtype=np.float64)
        self.params = np.ascontiguousarray(P)
        self._keep = [native.make_mesh_struct(m.as_abi_arrays()) for m in self.meshes]
        arr = (native.ZsmeMesh * self.n)(*[k[0] for k in self._keep])
        self._arr = arr
        self._st = self.settings.to_struct()
        h = ct.c_void_p()
        native.check(self.lib.zsme_batch_create(model.encode(), self.n, ct.addressof(arr), ct.addressof(self._st),
                                                _p(self.params), int(device), ct.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.zsme_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, i: int, q: np.ndarray, t: float = 0.0):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.meshes[i].n_cells, self.nq)
        native.check(self.lib.zsme_batch_set_state(self.h, int(i), _p(q), float(t)))

    def get_state(self, i: int) -> np.ndarray:
        q = np.empty((self.meshes[i].n_cells, self.nq))
        native.check(self.lib.zsme_batch_get_state(self.h, int(i), _p(q)))
        return q

    def time(self, i: int):
        t, d = ct.c_double(), ct.c_double()
        native.check(self.lib.zsme_batch_get_time(self.h, int(i), ct.byref(t), ct.byref(d)))
        return t.value, d.value

    def step(self, n: int = 1):
        native.check(self.lib.zsme_step(self.h, int(n)))

    def sync(self, check: bool = True) -> native.ZsmeDiag:
        d = native.ZsmeDiag()
        native.check(self.lib.zsme_get_diag(self.h, ct.byref(d)))
        if check:
            native.check(self.lib.zsme_sync(self.h))
        return d

    @property
    def stream(self) -> int:
        return self.lib.zsme_stream(self.h) or 0

    def set_profiling(self, on: bool = True):
        native.check(self.lib.zsme_set_profiling(self.h, int(bool(on))))

    def launches_per_step(self) -> int:
        n = ct.c_int32()
        native.check(self.lib.zsme_launches_per_step(self.h, ct.byref(n)))
        return n.value


LAUNCH_KEYS = ("prep", "face", "gather", "finalize", "prep_occ", "face_occ", "finalize_occ", "tile_faces",
               "fuse_final", "prep_lean")
LAUNCH_DEFAULTS = {"prep": 128, "face": 128, "gather": 128, "finalize": 128, "prep_occ": 1, "face_occ": 1,
                   "finalize_occ": 1, "tile_faces": 256, "fuse_final": 0, "prep_lean": 1}


def set_launch(h, cfg):
    """Launch configuration of a handle: dict with LAUNCH_KEYS (threads per
    block of each kernel, register caps as blocks per SM, tile_faces: 0 for
    the separate face and gather kernels, else the fused tile kernel's most
    faces per tile, fuse_final: the last stage's gather inside the finalize
    kernel, prep_lean: the lean face-state kernel); missing keys take
    LAUNCH_DEFAULTS."""
    lib = native.load()
    b = (ct.c_int32 * len(LAUNCH_KEYS))(*[int(cfg.get(k, LAUNCH_DEFAULTS[k])) for k in LAUNCH_KEYS])
    native.check(lib.zsme_set_launch(h, b))


def get_launch(h):
    lib = native.load()
    b = (ct.c_int32 * len(LAUNCH_KEYS))()
    native.check(lib.zsme_get_launch(h, b))
    return dict(zip(LAUNCH_KEYS, [int(x) for x in b]))
