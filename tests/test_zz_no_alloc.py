"""zsme_compute_dt_noalloc: the CFL step for callers that cannot allocate
device memory when they need it (memory reserved up front, fixed budgets).

It must give the same step as zsme_compute_dt (the allocating path that
keeps its partial minima in a cudaMalloc'd buffer), through the C ABI, on
two calls in a row -- the second call reuses the library's static scratch
array as the first left it.  This file is collected last on purpose.
"""
import ctypes as ct

import numpy as np
import pytest

from zoomy_dmplex_b200 import cases, models, native
from zoomy_dmplex_b200.solver import Solver

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _params(c):
    names, vals = models.parameter_table(c.model)
    for k, v in c.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


@pytest.mark.parametrize("make", [lambda: cases.level2(48), lambda: cases.plain_l0(60)])
def test_noalloc_dt_matches_compute_dt_twice(make):
    torch = pytest.importorskip("torch")
    c = make()
    p = _params(c)
    g = Solver(c.model, c.mesh, c.settings, p)
    g.set_state(c.q0)
    lib = native.load()
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    rc = dev(c.mesh.inradius_proxy())
    prm = dev(p)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    q_prev = None
    for call in range(2):
        if call == 1:
            g.step(3)                      # a different state for the second call
        q = dev(g.get_state())
        a = dev(g.get_aux())
        want = g.compute_dt()
        rcode = lib.zsme_compute_dt_noalloc(c.model.encode(), c.mesh.n_cells, q.data_ptr(), a.data_ptr(),
                                            rc.data_ptr(), prm.data_ptr(), c.settings.cfl, out.data_ptr(),
                                            ct.c_void_p(stream))
        assert rcode == 0, lib.zsme_last_error()
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= TOL * want, (call, got, want)
        if q_prev is not None:
            assert not torch.equal(q, q_prev)
        q_prev = q


def test_noalloc_rejects_oversize_and_bad_args():
    torch = pytest.importorskip("torch")
    lib = native.load()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = buf.data_ptr()
    rcode = lib.zsme_compute_dt_noalloc(b"sme2d_l2", (1 << 24) + 1, ptr, ptr, ptr, ptr, 0.45, ptr, None)
    assert rcode == 6 and b"exceed" in lib.zsme_last_error()
    assert lib.zsme_compute_dt_noalloc(b"nope", 1, ptr, ptr, ptr, ptr, 0.45, ptr, None) == 3
    assert lib.zsme_compute_dt_noalloc(b"sme2d_l2", 1, None, ptr, ptr, ptr, 0.45, ptr, None) == 1
