"""ctypes binding of the oracle (test infrastructure, the checker only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  ``Oracle`` mirrors the C ABI of the product (include/zsme.h) so
that a parity test drives both the same way.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "liboracle_ref.so")

FN = dict(numerical_flux=0, numerical_fluctuations=1, local_max_abs_eigenvalue=2, source=3,
          source_jacobian_wrt_variables=4, source_jacobian_wrt_aux_variables=5,
          update_variables=6, update_aux_variables=7, boundary_conditions=8, eigenvalues=9,
          flux=10, aux_jacobian=11, nonconservative_matrix=12)


def build(ref: bool = False):
    """Compile the oracle (and, with ref=True, the reference-header variant)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


_libs = {}


def load(ref: bool = False):
    path = REF_LIB if ref else LIB
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise FileNotFoundError(path + " is not built (make -C oracle%s)" % (" ref" if ref else ""))
    lib = ct.CDLL(path)
    P = ct.POINTER(ct.c_double)
    vp = ct.c_void_p
    lib.oracle_last_error.restype = ct.c_char_p
    lib.oracle_create.argtypes = [ct.c_char_p, vp, vp, P, ct.POINTER(vp)]
    lib.oracle_destroy.argtypes = [vp]
    lib.oracle_set_state.argtypes = [vp, P, ct.c_double]
    lib.oracle_get_state.argtypes = [vp, P]
    lib.oracle_get_aux.argtypes = [vp, P]
    lib.oracle_rhs.argtypes = [vp, ct.c_double, P, P]
    lib.oracle_gradient.argtypes = [vp, P, P]
    lib.oracle_update_state.argtypes = [vp]
    lib.oracle_source.argtypes = [vp, ct.c_double]
    lib.oracle_compute_dt.argtypes = [vp, P]
    lib.oracle_step.argtypes = [vp, ct.c_int]
    lib.oracle_step_dt.argtypes = [vp, ct.c_int, P]
    lib.oracle_get_time.argtypes = [vp, P, P]
    lib.oracle_set_params.argtypes = [vp, P]
    lib.oracle_newton_unconverged.argtypes = [vp]
    lib.oracle_mood_cells.argtypes = [vp]
    lib.oracle_mood_cells.restype = ct.c_longlong
    lib.oracle_set_threads.argtypes = [ct.c_int]
    lib.oracle_model_info.argtypes = [ct.c_char_p] + [ct.POINTER(ct.c_int)] * 4
    lib.oracle_pointwise.argtypes = [ct.c_char_p, ct.c_int, P, P, P, P, P, P, ct.c_double, P]
    lib.oracle_flux_vjp.argtypes = [ct.c_char_p, P, P, P, P, P, P, P, P]
    lib.oracle_create_counting.argtypes = [ct.c_char_p, vp, vp, P, ct.POINTER(vp)]
    lib.oracle_flop_counts.argtypes = [ct.POINTER(ct.c_longlong)]
    lib.oracle_implicit_function.argtypes = [vp, ct.c_double, P, P, P]
    lib.oracle_implicit_jacobian.argtypes = [vp, ct.c_double, P, ct.c_double, P, P]
    lib.oracle_implicit_stats.argtypes = [vp, ct.POINTER(ct.c_int)]
    _libs[path] = lib
    return lib


def _p(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def model_info(model: str, ref: bool = False):
    lib = load(ref)
    v = [ct.c_int() for _ in range(4)]
    rc = lib.oracle_model_info(model.encode(), *[ct.byref(x) for x in v])
    if rc:
        raise ValueError(lib.oracle_last_error().decode())
    return dict(n_dof_q=v[0].value, n_dof_qaux=v[1].value, n_parameters=v[2].value, dimension=v[3].value)


def pointwise(model: str, fn: str, qL, aL, p, n=None, qR=None, aR=None, s=0.0, ref=False):
    lib = load(ref)
    f = lambda a: np.ascontiguousarray(a if a is not None else np.zeros(16), dtype=np.float64)
    qL, aL, p = f(qL), f(aL), f(p)
    qR = f(qR if qR is not None else qL)
    aR = f(aR if aR is not None else aL)
    n = f(n if n is not None else np.array([1.0, 0.0, 0.0]))
    out = np.zeros(4096)
    k = lib.oracle_pointwise(model.encode(), FN[fn], _p(qL), _p(qR), _p(aL), _p(aR), _p(p), _p(n),
                             float(s), _p(out))
    if k < 0:
        raise ValueError(lib.oracle_last_error().decode())
    return out[:k].copy()


def face_jacobian(model: str, qL, qR, p, n, aL=None, aR=None):
    """d[numerical_flux, numerical_fluctuations] / d[qL, qR] by dual numbers:
    (3 nq) x (2 nq)."""
    lib = load(False)
    f = lambda a: np.ascontiguousarray(a if a is not None else np.zeros(16), dtype=np.float64)
    nq = len(qL)
    out = np.zeros(6 * nq * nq)
    k = lib.oracle_pointwise(model.encode(), 13, _p(f(qL)), _p(f(qR)), _p(f(aL)), _p(f(aR)), _p(f(p)), _p(f(n)),
                             0.0, _p(out))
    if k < 0:
        raise ValueError(lib.oracle_last_error().decode())
    return out.reshape(3 * nq, 2 * nq)


def flux_vjp(model: str, qL, qR, p, n, w, aL=None, aR=None):
    """g = w^T d[numerical_flux, numerical_fluctuations] / d[qL, qR] from the
    plugin's generated reverse sweep, or None if the plugin has none."""
    lib = load(False)
    f = lambda a: np.ascontiguousarray(a if a is not None else np.zeros(16), dtype=np.float64)
    g = np.zeros(2 * len(qL))
    k = lib.oracle_flux_vjp(model.encode(), _p(f(qL)), _p(f(qR)), _p(f(aL)), _p(f(aR)), _p(f(p)), _p(f(n)),
                            _p(f(w)), _p(g))
    return None if k < 0 else g[:k].copy()


def set_threads(n: int = 0, ref: bool = False) -> int:
    return load(ref).oracle_set_threads(n)


class Oracle:
    """CPU restatement of the reference step on one mesh (caller cell order)."""

    def __init__(self, model: str, mesh_abi: dict, settings_struct, params=None, ref=False):
        from zoomy_dmplex_b200 import native  # the zsme_mesh / zsme_settings layouts

        self.lib = load(ref)
        self.info = model_info(model, ref)
        self.nq = self.info["n_dof_q"]
        self.na = self.info["n_dof_qaux"]
        self.C = mesh_abi["n_cells"]
        self.F = mesh_abi["n_faces"]
        self._mesh_keep = native.make_mesh_struct(mesh_abi)
        self._settings = settings_struct
        h = ct.c_void_p()
        pp = None
        if params is not None:
            self._params = np.ascontiguousarray(params, dtype=np.float64)
            pp = _p(self._params)
        rc = self.lib.oracle_create(model.encode(), ct.addressof(self._mesh_keep[0]),
                                    ct.addressof(self._settings), pp, ct.byref(h))
        if rc:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def set_state(self, q, t=0.0):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.C, self.nq)
        self.lib.oracle_set_state(self.h, _p(q), float(t))

    def get_state(self):
        q = np.zeros((self.C, self.nq))
        self.lib.oracle_get_state(self.h, _p(q))
        return q

    def get_aux(self):
        a = np.zeros((self.C, self.na))
        self.lib.oracle_get_aux(self.h, _p(a))
        return a

    def rhs(self, x, t=0.0):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        f = np.zeros_like(x)
        self.lib.oracle_rhs(self.h, float(t), _p(x), _p(f))
        return f

    def gradient(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        dim = self.info["dimension"]
        g = np.zeros((self.C, self.nq * dim))
        self.lib.oracle_gradient(self.h, _p(x), _p(g))
        return g

    def update_state(self):
        self.lib.oracle_update_state(self.h)

    def implicit_function(self, x, xdot, t=0.0):
        """F(t, X, Xdot) = Xdot - S(X) - R(X) of the fully implicit strategy."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        xd = np.ascontiguousarray(xdot, dtype=np.float64).reshape(self.C, self.nq)
        f = np.zeros_like(x)
        self.lib.oracle_implicit_function(self.h, float(t), _p(x), _p(xd), _p(f))
        return f

    def implicit_jacobian(self, x, shift, t=0.0):
        """The implicit strategy's assembled matrix at (t, X, shift): diagonal
        blocks [C, nq, nq] and per face the (L, R) and (R, L) blocks [F, 2, nq, nq]."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.C, self.nq)
        d = np.zeros((self.C, self.nq, self.nq))
        o = np.zeros((self.F, 2, self.nq, self.nq))
        self.lib.oracle_implicit_jacobian(self.h, float(t), _p(x), float(shift), _p(d), _p(o))
        return d, o

    def implicit_stats(self):
        """Last implicit step: Newton iterations, GMRES iterations, halvings, stop reason."""
        v = (ct.c_int * 4)()
        self.lib.oracle_implicit_stats(self.h, v)
        return [int(x) for x in v]

    def source(self, dt):
        self.lib.oracle_source(self.h, float(dt))

    def compute_dt(self):
        d = ct.c_double()
        self.lib.oracle_compute_dt(self.h, ct.byref(d))
        return d.value

    def step(self, n=1, dts=None):
        if dts is None:
            self.lib.oracle_step(self.h, int(n))
        else:
            d = np.ascontiguousarray(dts, dtype=np.float64)
            self.lib.oracle_step_dt(self.h, int(d.size), _p(d))

    def time(self):
        t, d = ct.c_double(), ct.c_double()
        self.lib.oracle_get_time(self.h, ct.byref(t), ct.byref(d))
        return t.value, d.value

    def newton_unconverged(self):
        return self.lib.oracle_newton_unconverged(self.h)

    def mood_cells(self):
        """Cells redone at first order by MOOD over all steps so far."""
        return self.lib.oracle_mood_cells(self.h)


FLOP_PHASES = ("prep", "face", "gather", "final")
FLOP_OPS = ("add", "mul", "div", "sqrt", "other")


def flop_counts(model: str, mesh_abi: dict, settings_struct, params, q0, steps: int = 1, ref=False):
    """The floating-point operations of `steps` oracle steps from q0, counted
    by the Counted-scalar instance (flopcount.h): {phase: {op: count}} with
    phases prep / face / gather / final and ops add (+ and -), mul, div, sqrt,
    other (cbrt, pow).  set_state's constraints and initial dt are not in
    the count.  Runs the oracle on one thread (the counters are global) and
    restores all threads afterwards."""
    from zoomy_dmplex_b200 import native

    lib = load(ref)
    keep = native.make_mesh_struct(mesh_abi)
    pr = np.ascontiguousarray(params, dtype=np.float64)
    h = ct.c_void_p()
    if lib.oracle_create_counting(model.encode(), ct.addressof(keep[0]), ct.addressof(settings_struct), _p(pr),
                                  ct.byref(h)):
        raise RuntimeError(lib.oracle_last_error().decode())
    lib.oracle_set_threads(1)
    try:
        q = np.ascontiguousarray(q0, dtype=np.float64)
        lib.oracle_set_state(h, _p(q), 0.0)
        lib.oracle_flop_reset()
        lib.oracle_step(h, int(steps))
        out = (ct.c_longlong * (len(FLOP_PHASES) * len(FLOP_OPS)))()
        lib.oracle_flop_counts(out)
    finally:
        lib.oracle_destroy(h)
        lib.oracle_set_threads(0)
    v = list(out)
    n = len(FLOP_OPS)
    return {ph: dict(zip(FLOP_OPS, v[i * n:(i + 1) * n])) for i, ph in enumerate(FLOP_PHASES)}


class TangentOracle(Oracle):
    """The oracle on Dual<1> numbers: one tangent-linear direction (state and
    parameters) carried through the step (the branches are decided by the
    values, as in the plain run)."""

    def __init__(self, model: str, mesh_abi: dict, settings_struct, params=None, ref=False):
        from zoomy_dmplex_b200 import native

        self.lib = load(ref)
        self.lib.oracle_create_tlm.argtypes = [ct.c_char_p, ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_double),
                                               ct.POINTER(ct.c_void_p)]
        self.lib.oracle_set_tangent.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)]
        self.lib.oracle_get_tangent.argtypes = [ct.c_void_p, ct.POINTER(ct.c_double)]
        self.info = model_info(model, ref)
        self.nq = self.info["n_dof_q"]
        self.na = self.info["n_dof_qaux"]
        self.C = mesh_abi["n_cells"]
        self.F = mesh_abi["n_faces"]
        self._mesh_keep = native.make_mesh_struct(mesh_abi)
        self._settings = settings_struct
        h = ct.c_void_p()
        self._params = np.ascontiguousarray(params, dtype=np.float64) if params is not None else None
        pp = _p(self._params) if params is not None else None
        rc = self.lib.oracle_create_tlm(model.encode(), ct.addressof(self._mesh_keep[0]),
                                        ct.addressof(self._settings), pp, ct.byref(h))
        if rc:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        self.h = h

    def set_tangent(self, dq=None, dp=None):
        dq = np.zeros((self.C, self.nq)) if dq is None else np.ascontiguousarray(dq, dtype=np.float64)
        dp = np.zeros(self.info["n_parameters"]) if dp is None else np.ascontiguousarray(dp, dtype=np.float64)
        self._dq, self._dp = dq, dp
        self.lib.oracle_set_tangent(self.h, _p(dq), _p(dp))

    def get_tangent(self):
        out = np.zeros((self.C, self.nq))
        self.lib.oracle_get_tangent(self.h, _p(out))
        return out
