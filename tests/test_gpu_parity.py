"""GPU step (libzsme.so, through the C ABI) against the CPU oracle.

Bar: per-step relative L2 and relative max error of h and of every moment
<= 1e-12 (TOL).  The kernels are compiled without FMA contraction, so for
models whose plugins use only + - * / sqrt the two sides round identically
and the results are expected to be bit-identical; Manning friction calls
cbrt, whose last bit may differ between CUDA and glibc.
"""
import numpy as np
import pytest

import oracle_py as O
from zoomy_dmplex_b200 import cases, mesh as M, models
from zoomy_dmplex_b200.solver import Solver

TOL = 1e-12
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _threads():
    O.set_threads(0)


def params(model, d):
    names, vals = models.parameter_table(model)
    for k, v in d.items():
        vals[names.index(k)] = v
    return np.array(vals)


def pair(case, **kw):
    s = cases.default_settings(**kw)
    p = params(case.model, case.params)
    g = Solver(case.model, case.mesh, s, p)
    o = O.Oracle(case.model, case.mesh.as_abi_arrays(), s.to_struct(), p)
    g.set_state(case.q0)
    o.set_state(case.q0)
    return g, o


def errs(a, b):
    """per-variable relative L2 and relative max error of a vs reference b."""
    out = []
    for i in range(b.shape[1]):
        nb = np.linalg.norm(b[:, i])
        mb = np.abs(b[:, i]).max()
        e = a[:, i] - b[:, i]
        out.append((np.linalg.norm(e) / nb if nb > 0 else np.linalg.norm(e),
                    np.abs(e).max() / mb if mb > 0 else np.abs(e).max()))
    return np.array(out)


def assert_close(a, b, tol=TOL, what=""):
    e = errs(a, b)
    assert np.all(np.isfinite(a)), what
    assert e.max() <= tol, "%s: per-variable (relL2, relmax) = %s" % (what, e)


def case_1d():
    m = M.interval(np.linspace(-1.5, 1.5, 301))
    x = m.cell_centroid[:, 0]
    b = 0.2 * np.exp(-x ** 2 / 0.05)
    h = 1.0 - b + 0.1 * np.exp(-(x + 0.5) ** 2 / 0.01)
    q = np.stack([b, h, 0.3 * h], axis=1)
    return cases.Case("1d", "sme1d_l0_malpasset", m, q, cases.default_settings(),
                      dict(g=9.81, rho=1.0, nu=1.0, lambda_s=0.2, e_x=0.01), 50)


def small_cases():
    return {
        "l0": cases.plain_l0(40),
        "l1": cases.adjoint_l1(40),
        "l2": cases.level2(40),
        "l4": cases.roofline_l4(40),
        "1d": case_1d(),
        "mixed": cases.mixed_level2(24),      # triangles + quadrilaterals, empty face slots
    }


CASES = small_cases()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("order,grad", [(1, "least_squares"), (2, "least_squares"), (2, "green_gauss")])
def test_rhs_one_step_map(name, order, grad):
    c = CASES[name]
    g, o = pair(c, reconstruction_order=order, gradient=grad)
    rng = np.random.default_rng(5)
    x = c.q0.copy()
    x[:, 2:] += 0.05 * rng.standard_normal(x[:, 2:].shape) * x[:, 1:2]
    fg, fo = g.rhs(x), o.rhs(x)
    assert_close(fg, fo, what="rhs %s o%d %s" % (name, order, grad))


@pytest.mark.parametrize("name", ["l2", "l4", "1d", "mixed"])
def test_rhs_bitwise_without_cbrt(name):
    """No FMA contraction + IEEE sqrt/div: identical rounding."""
    c = CASES[name]
    g, o = pair(c)
    x = c.q0.copy()
    x[:, 2] += 0.01
    assert np.array_equal(g.rhs(x), o.rhs(x))


@pytest.mark.parametrize("name", list(CASES))
def test_constraints_source_dt(name):
    c = CASES[name]
    g, o = pair(c)
    assert_close(g.get_state(), o.get_state(), what="set_state constraints")
    assert_close(g.get_aux(), o.get_aux(), what="aux")
    dg, do = g.compute_dt(), o.compute_dt()
    assert abs(dg - do) <= TOL * do
    g.source(5e-3)
    o.source(5e-3)
    assert_close(g.get_state(), o.get_state(), what="source")
    g.update_state()
    o.update_state()
    assert_close(g.get_state(), o.get_state(), what="update_state")


@pytest.mark.parametrize("name,steps", [("l0", 200), ("l1", 60), ("l2", 60), ("l4", 30), ("1d", 100),
                                        ("mixed", 60)])
def test_trajectory_per_step(name, steps):
    """Free-running oracle; the GPU takes the oracle's dt each step; every
    step is compared."""
    c = CASES[name]
    g, o = pair(c)
    worst = 0.0
    for k in range(steps):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        qg, qo = g.get_state(), o.get_state()
        e = errs(qg, qo).max()
        worst = max(worst, e)
        assert e <= TOL, "step %d: %g" % (k, e)
        assert qg[:, 1].min() >= 0.0
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0


@pytest.mark.parametrize("name", ["l0", "l2"])
def test_free_running_dt_and_state(name):
    """Both sides choose their own CFL dt (device-side reduction, CUDA graph)."""
    c = CASES[name]
    g, o = pair(c)
    n = 50
    g.step(n)
    o.step(n)
    tg, dtg = g.time()
    to, dto = o.time()
    assert abs(tg - to) <= TOL * to and abs(dtg - dto) <= TOL * dto
    assert_close(g.get_state(), o.get_state(), what="free run")


def test_t_end_landing():
    c = CASES["l0"]
    s = cases.default_settings(t_end=0.0123)
    p = params(c.model, c.params)
    g = Solver(c.model, c.mesh, s, p)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), s.to_struct(), p)
    g.set_state(c.q0)
    o.set_state(c.q0)
    g.step(500)           # steps past t_end are no-ops
    o.step(500)
    assert g.time()[0] == pytest.approx(0.0123, abs=1e-15)
    assert_close(g.get_state(), o.get_state(), what="t_end")


def test_deterministic_bitwise():
    c = CASES["l4"]
    outs = []
    for _ in range(2):
        g, _o = pair(c)
        g.step(10)
        outs.append(g.get_state())
    assert np.array_equal(outs[0], outs[1])


def test_lake_at_rest_first_order_gpu():
    c = cases.plain_l0(40)
    c.q0[:, 1] = 1.0 - c.q0[:, 0]
    g, _ = pair(c, reconstruction_order=1)
    g.step(50)
    q = g.get_state()
    assert np.abs(q[:, 0] + q[:, 1] - 1.0).max() < 1e-14
    assert np.abs(q[:, 2:]).max() < 1e-14


def test_config0_full_run():
    """Configuration 0 as specified: 60x60 jittered grid, least-squares
    gradients with Barth-Jespersen (Vacuum + TVD) limiting, Manning friction,
    200 steps, every step against the oracle (its dt imposed).  Manning's
    cbrt may round differently in CUDA and glibc, so the bar is the 1e-12
    tolerance rather than bit equality."""
    c = cases.plain_l0(60)
    assert c.settings.gradient == "least_squares" and c.steps == 200
    p = params(c.model, c.params)
    g = Solver(c.model, c.mesh, c.settings, p)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), p)
    g.set_state(c.q0)
    o.set_state(c.q0)
    for k in range(c.steps):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        assert_close(g.get_state(), o.get_state(), what="config 0 step %d" % (k + 1))
    q = g.get_state()
    assert q[:, 1].min() >= 0
    vol = c.mesh.cell_volume
    assert abs((q[:, 1] * vol).sum() - (c.q0[:, 1] * vol).sum()) < 1e-13
    # the same 200 steps free running (device CFL dt, CUDA graph)
    g2 = Solver(c.model, c.mesh, c.settings, p)
    o2 = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), p)
    g2.set_state(c.q0)
    o2.set_state(c.q0)
    g2.step(c.steps)
    o2.step(c.steps)
    assert_close(g2.get_state(), o2.get_state(), what="config 0 free run")
    assert abs(g2.time()[0] - o2.time()[0]) <= TOL * o2.time()[0]


def test_config1_full_run_per_step():
    """Configuration 1 as specified: SME level 2 on the 240x240 jittered
    grid, 500 steps, every step against the oracle (its dt imposed), bit for
    bit -- the level-2 plugins call no cbrt."""
    c = cases.level2(240)
    g, o = pair(c)
    for k in range(500):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        assert np.array_equal(g.get_state(), o.get_state()), "step %d" % k
    q = g.get_state()
    assert q[:, 1].min() >= 0
    d = g.sync()
    assert d.n_nonfinite == 0 and d.n_negative_depth == 0


def test_device_pointer_state_roundtrip():
    torch = pytest.importorskip("torch")
    c = CASES["l2"]
    g, _ = pair(c)
    t = torch.tensor(c.q0, dtype=torch.float64, device="cuda")
    g.set_state_device(t.data_ptr())
    out = torch.empty_like(t)
    g.get_state_device(out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), g.get_state())


@pytest.mark.parametrize("tile_faces", [0, 128])
def test_profile_kinds_per_step(tile_faces):
    """Per-kernel timing attributes every launch of a step to its own kind:
    two SSP stages (prep, flux and, with the separate kernels, gather each;
    the fused tile kernel counts as flux), finalize and its fallback, the
    step ends; launches_per_step counts the same kernels."""
    from zoomy_dmplex_b200.solver import set_launch

    c = CASES["l2"]
    g, _ = pair(c)
    set_launch(g.h, {"tile_faces": tile_faces})
    g.set_profiling(True)
    g.step(2)
    g.sync()
    prof = g.read_profile()
    g.set_profiling(False)
    n = {k: v[1] for k, v in prof.items()}
    assert n == {"begin_step": 2, "prep": 4, "flux": 4, "finalize": 2, "end_step": 2,
                 "gather": 0 if tile_faces else 4, "finalize_fallback": 2, "mood": 0}
    assert all(v[0] > 0 for k, v in prof.items() if n[k])
    assert g.launches_per_step() == sum(n.values()) // 2


def test_async_state_io_matches_blocking_calls():
    """Three independent one-step problems pipelined through the asynchronous
    state calls (page-locked host buffers, copies on their own streams) give
    the blocking calls' results bit for bit."""
    import torch

    c = CASES["l2"]
    g, _ = pair(c)
    qs = []
    for k in range(3):
        q = c.q0.copy()
        q[:, 2:] += 0.01 * k * q[:, 1:2]
        qs.append(q)
    ref = []
    for q in qs:
        g.set_state(q)
        g.step(1)
        ref.append(g.get_state())
    ins = [torch.from_numpy(q).pin_memory() for q in qs]
    outs = [torch.zeros(c.q0.shape, dtype=torch.float64).pin_memory() for _ in qs]
    for k in range(3):
        g.set_state_async(ins[k].data_ptr(), 0.0)
        g.step(1)
        g.get_state_async(outs[k].data_ptr())
    g.stream_wait_copies()
    g.sync()
    for k in range(3):
        assert np.array_equal(outs[k].numpy(), ref[k]), k
    assert np.array_equal(g.get_state(), ref[2])


def test_failure_detection_without_a_fault():
    """Health counters and zsme_sync's error: negative depths from the
    limited step at CFL 1.5 on a wet/dry patchwork, and a non-finite value
    planted in the state, are counted on the device and reported by
    zsme_sync as ZSME_ERR_STATE; the handle stays usable."""
    from zoomy_dmplex_b200.native import ZsmeError

    c = cases.wet_dry_patchwork(24)
    g = Solver(c.model, c.mesh, c.settings, params(c.model, c.params))
    g.set_state(c.q0)
    g.step(20)
    d = g.sync(check=False)
    assert d.n_negative_depth > 0 and d.n_nonfinite == 0
    with pytest.raises(ZsmeError, match="negative-depth"):
        g.sync()
    # a non-finite depth survives the constraints (a non-finite momentum does
    # not: the clamp max(-t, min(hu, t)), written as std::max / std::min
    # selects, returns its bound for NaN, as in the reference)
    q = c.q0.copy()
    q[7, 1] = np.nan
    g.set_state(q)
    g.step(1)
    d = g.sync(check=False)
    assert d.n_nonfinite > 0
    with pytest.raises(ZsmeError, match="non-finite"):
        g.sync()
    g.set_state(c.q0)                    # the handle is usable again
    g.step(1)
    assert np.all(np.isfinite(g.get_state()))


def test_fp64_fma_peak_is_measured():
    """zsme_fp64_fma_peak times FMA chains on every SM; a B200's FP64 rate
    lies in the tens of TFLOP/s."""
    import ctypes as ct

    from zoomy_dmplex_b200 import native

    v = ct.c_double()
    native.check(native.load().zsme_fp64_fma_peak(0, ct.byref(v)))
    assert 5.0 < v.value < 200.0, v.value


def test_newton_fast_path_coverage():
    """Which cells leave the Newton register fast path for the generic
    elimination (zsme_diag.n_newton_deferred): none for the generated
    plugins, whose sources do not depend on the aux variables (Manning
    friction on level 0, Navier slip on level 2, the 1-D model's slip)."""
    for c in (cases.plain_l0(30), cases.level2(30), case_1d()):
        g, _ = pair(c)
        g.step(3)
        d = g.sync()
        assert d.n_newton_deferred == 0, (c.name, d.n_newton_deferred)


@pytest.mark.parametrize("prep_lean", [0, 2, 3, 4])
@pytest.mark.parametrize("name", ["l2", "l4", "1d", "mixed"])
@pytest.mark.parametrize("grad", ["green_gauss", "least_squares"])
def test_face_state_kernels_bitwise(prep_lean, name, grad):
    """The order-2 face-state kernels (prep_lean 0: plain, 1: lean, 2..4: lean
    split over that many threads per cell) give the same RHS as the oracle bit
    for bit, and the same steps as the default kernel bit for bit."""
    from zoomy_dmplex_b200.solver import set_launch

    c = CASES[name]
    g, o = pair(c, gradient=grad)
    ref, _ = pair(c, gradient=grad)
    set_launch(g.h, {"prep_lean": prep_lean, "tile_faces": 0})
    set_launch(ref.h, {"prep_lean": 1, "tile_faces": 0})
    x = c.q0.copy()
    x[:, 2] += 0.01
    assert np.array_equal(g.rhs(x), o.rhs(x))
    for k in range(8):
        _, dt = o.time()
        o.step(1)
        g.step(1, dts=[dt])
        ref.step(1, dts=[dt])
        qg = g.get_state()
        assert np.array_equal(qg, ref.get_state()), k
        assert errs(qg, o.get_state()).max() <= TOL, k
