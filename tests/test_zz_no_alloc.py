"""zsme_compute_dt_noalloc: the CFL step for callers that cannot allocate
device memory when they need it (memory reserved up front, fixed budgets).

It must give the same step as zsme_compute_dt (the allocating path that
keeps its partial minima in a cudaMalloc'd buffer), through the C ABI, on
two calls in a row -- the second call reuses the library's static scratch
array as the first left it.  The cases cover every compiled model, a mesh
large enough that the final reduction loops over more than 256 partial
minima, a NaN depth planted in one cell (that cell alone drops out of the
minimum, as in the allocating path), and cells whose d_rc is >= DBL_MAX,
which the entry point leaves out of the minimum.  This file is collected
last on purpose.
"""
import ctypes as ct

import numpy as np
import pytest

from zoomy_dmplex_b200 import cases, mesh as meshmod, models, native
from zoomy_dmplex_b200.solver import Solver

pytestmark = pytest.mark.gpu
TOL = 1e-12
DBL_MAX = np.finfo(np.float64).max


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def _case_1d():
    x = np.linspace(0.0, 1.0, 401)
    xc = 0.5 * (x[1:] + x[:-1])
    q = np.zeros((xc.size, 3))
    q[:, 1] = 1.0 + 0.1 * np.exp(-((xc - 0.4) ** 2) / 0.01)
    q[:, 2] = 0.2 * q[:, 1]
    return cases.Case("line", "sme1d_l0_malpasset", meshmod.interval(x), q, cases.default_settings(), {}, 10)


CASES = {
    "sme2d_l2_48": lambda: cases.level2(48),
    "sme2d_l0_60": lambda: cases.plain_l0(60),
    "sme2d_l1_40": lambda: cases.adjoint_l1(40),
    "sme2d_l4_40": lambda: cases.roofline_l4(40),
    "sme1d_l0_400": _case_1d,
    # 79,202 cells: 310 partial minima, so the final kernel's strided loop runs
    "sme2d_l2_200": lambda: cases.level2(200),
}


class _Call:
    def __init__(self, c, p):
        self.torch = pytest.importorskip("torch")
        self.c = c
        self.lib = native.load()
        self.prm = self.dev(p)
        self.out = self.torch.full((1,), -1.0, dtype=self.torch.float64, device="cuda")

    def dev(self, a):
        return self.torch.tensor(np.ascontiguousarray(a), dtype=self.torch.float64, device="cuda")

    def __call__(self, q, a, rc):
        stream = self.torch.cuda.current_stream().cuda_stream
        qd, ad, rcd = self.dev(q), self.dev(a), self.dev(rc)
        rcode = self.lib.zsme_compute_dt_noalloc(self.c.model.encode(), len(rc), qd.data_ptr(),
                                                 ad.data_ptr(), rcd.data_ptr(), self.prm.data_ptr(),
                                                 self.c.settings.cfl, self.out.data_ptr(), ct.c_void_p(stream))
        assert rcode == 0, self.lib.zsme_last_error()
        self.torch.cuda.synchronize()
        return float(self.out.item())


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_dt_matches_compute_dt_twice(name):
    c = CASES[name]()
    p = _params(c)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    call = _Call(c, p)
    rc = c.mesh.inradius_proxy()
    q_prev = None
    for k in range(2):
        if k == 1:
            g.step(3)                      # a different state for the second call
        q = g.get_state()
        want = g.compute_dt()
        got = call(q, g.get_aux(), rc)
        assert abs(got - want) <= TOL * want, (k, got, want)
        if q_prev is not None:
            assert not np.array_equal(q, q_prev)
        q_prev = q


def test_noalloc_nan_depth_drops_only_that_cell():
    """A NaN depth in one cell: that cell has no wave speed and drops out of
    the minimum (VirtualSolver.hpp:320-326); every other cell still counts,
    in the allocating and the allocation-free path alike."""
    c = cases.level2(48)
    p = _params(c)
    g = Solver(c.model, c.mesh, c.settings, p)
    q0 = c.q0.copy()
    rc = c.mesh.inradius_proxy()
    # plant the NaN in the cell that sets the minimum, so a masked minimum would show
    g.set_state(q0)
    lam = np.abs(q0[:, 2] / q0[:, 1]) + np.sqrt(9.81 * q0[:, 1])
    worst = int(np.argmin(rc / lam))
    q0[worst, 1] = np.nan
    g.set_state(q0)
    q, a = g.get_state(), g.get_aux()
    assert np.isnan(q[worst, 1])
    want = g.compute_dt()
    got = _Call(c, p)(q, a, rc)
    assert np.isfinite(want) and abs(got - want) <= TOL * want, (got, want)
    # the same as the minimum over the other cells alone
    rc_skip = rc.copy()
    rc_skip[worst] = DBL_MAX
    assert abs(_Call(c, p)(q, a, rc_skip) - want) <= TOL * want


def test_noalloc_skips_cells_with_rc_at_dbl_max():
    """Cells whose d_rc is >= DBL_MAX (or +inf) do not constrain the step:
    the way a partitioned caller keeps its halo cells out of the minimum.
    The cells may come in any order and any number, so one cell alone is a
    valid input."""
    c = cases.level2(48)
    p = _params(c)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    q, a = g.get_state(), g.get_aux()
    rc = c.mesh.inradius_proxy()
    call = _Call(c, p)
    full = call(q, a, rc)
    # with every cell but one excluded (DBL_MAX or +inf), the step is that
    # cell's own, as computed on a one-cell input
    keep = 17
    rc_one = np.full_like(rc, DBL_MAX)
    rc_one[::2] = np.inf
    rc_one[keep] = rc[keep]
    one = call(q, a, rc_one)
    assert one >= full
    alone = call(q[keep:keep + 1], a[keep:keep + 1], rc[keep:keep + 1])
    assert one == alone, (one, alone)
    # with every cell excluded, no cell constrains: the model's dt_max
    none = call(q, a, np.full_like(rc, DBL_MAX))
    assert none > one


def test_noalloc_rejects_oversize_and_bad_args():
    torch = pytest.importorskip("torch")
    lib = native.load()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = buf.data_ptr()
    rcode = lib.zsme_compute_dt_noalloc(b"sme2d_l2", (1 << 24) + 1, ptr, ptr, ptr, ptr, 0.45, ptr, None)
    assert rcode == 6 and b"exceed" in lib.zsme_last_error()
    assert lib.zsme_compute_dt_noalloc(b"nope", 1, ptr, ptr, ptr, ptr, 0.45, ptr, None) == 3
    assert lib.zsme_compute_dt_noalloc(b"sme2d_l2", 1, None, ptr, ptr, ptr, 0.45, ptr, None) == 1
