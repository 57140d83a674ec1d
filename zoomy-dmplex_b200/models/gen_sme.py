#!/usr/bin/env python
"""Generator of the shallow-water-moment (SME) model plugins.

The reference ships its model as two generated headers, ``Model.H`` and
``Numerics.H`` (reference ``Model.H:29-398``, ``Numerics.H:29-109``), produced
by a sympy pipeline (``create_model.py:80-101``) that is not available here.
This script derives the same plugin interface from the SME equations itself
(Kowalski & Torrilhon 2019, "Moment approximations and model cascades for
shallow flow") with sympy and prints C++ with identical function names,
signatures and conventions:

* state ``Q = [b, h, hu_0..hu_L (, hv_0..hv_L)]`` with ``idx_b = 0``,
  ``idx_h = 1``; ``hu_0`` is the depth-averaged momentum, ``hu_j`` (j>=1) the
  moment ``h*alpha_j`` of the Legendre ansatz ``u = u_m + sum_j alpha_j phi_j``;
* ``numerical_flux`` = central flux of the hydrostatically reconstructed states
  ``q*`` (Audusse), ``numerical_fluctuations`` = Rusanov dissipation on ``q*``
  plus the hydrostatic-reconstruction pressure correction plus the midpoint
  path integral of the moment non-conservative product; the first ``n_dof_q``
  entries go into the right cell, the last ``n_dof_q`` into the left cell
  (reference ``TransportStep.hpp:461-466``);
* ``update_variables`` = the wet/dry momentum clamp, ``update_aux_variables`` =
  the Kurganov-Petrova regularised ``1/h`` (reference ``Model.H:195-222``);
* ``boundary_conditions`` index 0 = wall (normal component of every momentum
  pair reflected, reference ``Model.H:356-375``).

Variants:

* ``sme2d_l<L>`` -- 2-D SME level L, aux ``[hinv]``, parameters
  ``g, nu, lambda, n_manning, e_x, e_y``; source = Navier-slip bottom friction
  with slip length ``lambda`` and viscous moment damping ``nu`` plus Manning
  friction on the mean momentum plus the slope forcing ``e``;
* ``sme1d_l0_malpasset`` -- the 1-D level-0 model with the same parameter
  names, aux layout and source law as the reference's shipped ``Model.H``
  (``Model.H:31-44,110-123``); it exists to pin this generator against the
  reference's own generated header.

Usage: ``python gen_sme.py [--out DIR] [name ...]`` (default: all variants).
"""
import argparse
import os
import sys

import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))

# --------------------------------------------------------------------------
# Legendre moment coefficients on the scaled vertical coordinate zeta in [0,1]
# (zeta = 0 at the bed; phi_j(0) = 1).
# --------------------------------------------------------------------------
_z = sp.Symbol("zeta")


def phi(j):
    return sp.expand(sp.legendre(j, 1 - 2 * _z))


def moment_coefficients(L):
    """A_ijk, B_ijk, C_ij of Kowalski & Torrilhon (exact rationals)."""
    ph = [phi(j) for j in range(L + 1)]
    dph = [sp.diff(f, _z) for f in ph]
    Ph = [sp.integrate(f, (_z, 0, _z)) for f in ph]
    A = {}
    B = {}
    C = {}
    for i in range(1, L + 1):
        for j in range(1, L + 1):
            C[i, j] = sp.integrate(dph[i] * dph[j], (_z, 0, 1))
            # (2i+1) int phi_i' Phi_j = -delta_ij  (sanity of the basis)
            chk = (2 * i + 1) * sp.integrate(dph[i] * Ph[j], (_z, 0, 1))
            assert chk == (-1 if i == j else 0), (i, j, chk)
            for k in range(1, L + 1):
                A[i, j, k] = (2 * i + 1) * sp.integrate(ph[i] * ph[j] * ph[k], (_z, 0, 1))
                B[i, j, k] = (2 * i + 1) * sp.integrate(dph[i] * Ph[j] * ph[k], (_z, 0, 1))
    for j in range(L + 1):
        assert sp.integrate(ph[j] * ph[j], (_z, 0, 1)) == sp.Rational(1, 2 * j + 1)
        assert ph[j].subs(_z, 0) == 1
    return A, B, C


# --------------------------------------------------------------------------
# C++ printer (generated-header style: std:: maths, (T) casts inside max/min)
# --------------------------------------------------------------------------
def _num(x):
    if isinstance(x, sp.Integer) or (isinstance(x, sp.Rational) and x.q == 1):
        return "%d.0" % int(x)
    if isinstance(x, sp.Rational):
        return "(%d.0/%d.0)" % (x.p, x.q)
    return repr(float(x))


class Printer:
    def __init__(self, T="T"):
        self.T = T

    def p(self, e):
        e = sp.sympify(e)
        if e.is_Symbol:
            return e.name
        if e.is_Number:
            s = _num(e)
            return "(" + s + ")" if s.startswith("-") else s
        if isinstance(e, sp.Add):
            terms = list(e.args)
            out = self.p(terms[0])
            for t in terms[1:]:
                c, rest = t.as_coeff_Mul()
                if c.is_Number and c < 0:
                    out += " - " + self.p(-t)
                else:
                    out += " + " + self.p(t)
            return "(" + out + ")"
        if isinstance(e, sp.Mul):
            c, rest = e.as_coeff_Mul()
            if c.is_Number and c < 0:
                return "(-" + self.p(-e) + ")"
            num, den = [], []
            for a in e.args:
                if isinstance(a, sp.Pow) and a.exp.is_Number and a.exp < 0:
                    den.append(sp.Pow(a.base, -a.exp, evaluate=False))
                elif a.is_Rational and not a.is_Integer:
                    # rational coefficient -> multiplication by its double
                    # (an IEEE division by a constant costs a full sequence)
                    num.insert(0, sp.Float(float(a), 17))
                else:
                    num.append(a)
            ns = "*".join(self.p(a) for a in num) if num else "1.0"
            if not den:
                return ns
            ds = "*".join(self.p(a) for a in den)
            if len(den) > 1:
                ds = "(" + ds + ")"
            return "(" + ns + "/" + ds + ")"
        if isinstance(e, sp.Pow):
            b, x = e.base, e.exp
            bs = self.p(b)
            if x.is_Integer:
                n = int(x)
                if n < 0:
                    return "(1.0/" + self.p(sp.Pow(b, -n, evaluate=False)) + ")"
                if n == 0:
                    return "1.0"
                return "(" + "*".join([bs] * n) + ")"
            if x == sp.Rational(1, 2):
                return "std::sqrt(" + bs + ")"
            if x == sp.Rational(-1, 2):
                return "(1.0/std::sqrt(" + bs + "))"
            if x.is_Rational and x.q == 2 and x > 0:
                k = (x.p - 1) // 2
                return "(" + "*".join([bs] * k + ["std::sqrt(" + bs + ")"]) + ")"
            if x == sp.Rational(1, 3):
                return "std::cbrt(" + bs + ")"
            if x == sp.Rational(-1, 3):
                return "(1.0/std::cbrt(" + bs + "))"
            if x.is_Rational and x.q == 3:
                # b^(m + r/3) = b*...*b * cbrt(b)^r: one cube root, shared by every
                # such power of b after the compiler's CSE, instead of a pow each
                if x < 0:
                    return "(1.0/" + self.p(sp.Pow(b, -x, evaluate=False)) + ")"
                m, r = divmod(int(x.p), 3)
                return "(" + "*".join([bs] * m + ["std::cbrt(" + bs + ")"] * r) + ")"
            return "std::pow(" + bs + ", " + _num(x) + ")"
        if isinstance(e, (sp.Max, sp.Min)):
            fn = "std::max" if isinstance(e, sp.Max) else "std::min"
            args = list(e.args)
            # numbers first, like the reference printer: std::max((T)eps, x)
            args.sort(key=lambda a: 0 if a.is_Number else 1)
            s = self._arg(args[-1])
            for a in reversed(args[:-1]):
                s = "%s(%s, %s)" % (fn, self._arg(a), s)
            return s
        if isinstance(e, sp.Abs):
            return "std::fabs(" + self.p(e.args[0]) + ")"
        if isinstance(e, Sel):
            a, b, x, y = e.args
            return "((%s < %s) ? %s : %s)" % (self._arg(a), self._arg(b), self._arg(x), self._arg(y))
        if isinstance(e, SelNZ):
            a, x, y = e.args
            return "((%s != %s) ? %s : %s)" % (self._arg(a), self._arg(sp.Integer(0)), self._arg(x), self._arg(y))
        if isinstance(e, sp.Heaviside):
            h0 = e.args[1] if len(e.args) > 1 else sp.Rational(1, 2)
            return "Heaviside(" + self.p(e.args[0]) + ", " + _num(h0) + ")"
        raise NotImplementedError(type(e), e)

    def _arg(self, a):
        if a.is_Number:
            return "(%s)%s" % (self.T, _num(a))
        return self.p(a)


def emit_body(exprs, res_name="res", size=None, indent="    "):
    """CSE the outputs and print `T tK = ...; res[i] = ...;` lines."""
    exprs = [sp.sympify(e) for e in exprs]
    size = size if size is not None else len(exprs)
    syms = sp.numbered_symbols("t")
    repl, red = sp.cse(exprs, symbols=syms, optimizations="basic")
    pr = Printer()
    lines = []
    for s, e in repl:
        lines.append("%sT %s = %s;" % (indent, s.name, pr.p(e)))
    lines.append("%sSimpleArray<T, %d> %s;" % (indent, size, res_name))
    for i, e in enumerate(red):
        lines.append("%s%s[%d] = %s;" % (indent, res_name, i, pr.p(e)))
    lines.append("%sreturn %s;" % (indent, res_name))
    return "\n".join(lines)


def arr(name, n):
    return [sp.Symbol("%s[%d]" % (name, i)) for i in range(n)]


# --------------------------------------------------------------------------
# Reverse-mode derivatives (vector-Jacobian products) of printed code
# --------------------------------------------------------------------------
class Sel(sp.Function):
    """Sel(a, b, x, y) = (a < b) ? x : y, printed as a conditional."""
    nargs = 4


class SelNZ(sp.Function):
    """SelNZ(a, x, y) = (a != 0) ? x : y, printed as a conditional."""
    nargs = 3


def _vjp(e, a, acc):
    """Add the adjoint a of expression e to its leaf symbols (acc: symbol ->
    list of terms).  The rules differentiate the C++ this module's Printer
    emits for e, with the conventions of the dual numbers (csrc/dual.h): a
    max / min takes the derivative of the argument std::max / std::min
    returns (the first one on a tie), d|x| = +dx at x = 0, and a square or
    cube root has a zero derivative where it is 0."""
    if e.is_Symbol:
        acc.setdefault(e, []).append(a)
    elif e.is_Number:
        return
    elif isinstance(e, sp.Add):
        for t in e.args:
            _vjp(t, a, acc)
    elif isinstance(e, sp.Mul):
        args = e.args
        for i, f in enumerate(args):
            if not f.is_Number:
                _vjp(f, a * sp.Mul(*(args[:i] + args[i + 1:])), acc)
    elif isinstance(e, sp.Pow):
        b, x = e.base, e.exp
        if x.is_Integer:
            _vjp(b, a * x * b ** (x - 1), acc)
        elif x == sp.Rational(1, 2):                       # std::sqrt(b)
            _vjp(b, a * Sel(0, e, sp.Rational(1, 2) / e, 0), acc)
        elif x == sp.Rational(-1, 2):                      # 1.0/std::sqrt(b)
            s = sp.sqrt(b)
            _vjp(b, -a * e ** 2 * Sel(0, s, sp.Rational(1, 2) / s, 0), acc)
        elif x.is_Rational and x.q == 2 and x > 0:         # b*...*b*std::sqrt(b)
            k = (x.p - 1) // 2
            s = sp.sqrt(b)
            _vjp(b, a * (k * b ** (k - 1) * s + b ** k * Sel(0, s, sp.Rational(1, 2) / s, 0)), acc)
        elif x == sp.Rational(1, 3):                       # std::cbrt(b)
            _vjp(b, a * SelNZ(e, 1 / (3 * e * e), 0), acc)
        elif x == sp.Rational(-1, 3):                      # 1.0/std::cbrt(b)
            c = sp.cbrt(b)
            _vjp(b, -a * e ** 2 * SelNZ(c, 1 / (3 * c * c), 0), acc)
        elif x.is_Rational and x.q == 3 and x > 0:         # b*...*b*cbrt(b)^r
            m, r = divmod(int(x.p), 3)
            c = sp.cbrt(b)
            dc = SelNZ(c, 1 / (3 * c * c), 0)
            _vjp(b, a * (m * b ** (m - 1) * c ** r + b ** m * r * c ** (r - 1) * dc), acc)
        elif x.is_Rational and x.q == 3:                   # 1.0/(b*...*b*cbrt(b)^r)
            _vjp(sp.Pow(b, -x, evaluate=False), -a * e ** 2, acc)
        else:                                              # std::pow(b, x)
            _vjp(b, a * SelNZ(b, x * b ** (x - 1), 0), acc)
    elif isinstance(e, (sp.Max, sp.Min)):
        args = sorted(e.args, key=lambda t: 0 if t.is_Number else 1)    # the printer's nesting
        _vjp_minmax(isinstance(e, sp.Max), args, a, acc)
    elif isinstance(e, sp.Abs):                            # std::fabs(x)
        x = e.args[0]
        _vjp(x, Sel(x, 0, -a, a), acc)
    elif isinstance(e, sp.Heaviside):
        return
    else:
        raise NotImplementedError(type(e), e)


def _vjp_minmax(is_max, args, a, acc):
    # fn(args[0], fn(args[1], ... fn(args[-2], args[-1])))
    if len(args) == 1:
        _vjp(args[0], a, acc)
        return
    x, rest = args[0], args[1:]
    y = rest[0] if len(rest) == 1 else (sp.Max if is_max else sp.Min)(*rest, evaluate=False)
    if is_max:      # std::max(x, y) = (x < y) ? y : x
        _vjp(x, Sel(x, y, 0, a), acc)
        _vjp_minmax(True, rest, Sel(x, y, a, 0), acc)
    else:           # std::min(x, y) = (y < x) ? y : x
        _vjp(x, Sel(y, x, 0, a), acc)
        _vjp_minmax(False, rest, Sel(y, x, a, 0), acc)


def emit_vjp_body(exprs, inputs, w_name="w", g_name="g", indent="    "):
    """g[j] = sum_k w[k] d exprs[k] / d inputs[j]: the outputs' SSA (CSE)
    followed by its reverse sweep, one adjoint per SSA value."""
    exprs = [sp.sympify(e) for e in exprs]
    w = arr(w_name, len(exprs))
    repl, red = sp.cse(exprs, symbols=sp.numbered_symbols("t"), optimizations="basic")
    acc = {}
    for k, e in enumerate(red):
        _vjp(e, w[k], acc)
    adj = []
    for s, e in reversed(repl):
        terms = acc.pop(s, [])
        if not terms:
            continue
        a_s = sp.Symbol("a_" + s.name)
        adj.append((a_s, sp.Add(*terms)))
        _vjp(e, a_s, acc)
    pr = Printer()
    lines = ["%sT %s = %s;" % (indent, s.name, pr.p(e)) for s, e in repl]
    lines += ["%sT %s = %s;" % (indent, s.name, pr.p(e)) for s, e in adj]
    for j, x in enumerate(inputs):
        lines.append("%s%s[%d] = %s;" % (indent, g_name, j, pr.p(sp.Add(*acc.get(x, [])))))
    return "\n".join(lines)


# --------------------------------------------------------------------------
# Model specification
# --------------------------------------------------------------------------
class Spec:
    def __init__(self, name, dim, L, variant):
        self.name, self.dim, self.L, self.variant = name, dim, L, variant
        nmom = L + 1
        self.nmom = nmom
        self.n_q = 2 + dim * nmom
        if variant == "malpasset":
            self.aux_names = ["dq0dx", "dhdx", "dbdx", "hinv"]
            self.ihinv = 3
            self.params = ["g", "rho", "nu", "lambda_s", "e_x"]
            self.defaults = [9.81, 1.0, 1.0, 0.5, 0.0]
        else:
            self.aux_names = ["hinv"]
            self.ihinv = 0
            self.params = ["g", "nu", "lambda", "n_manning", "e_x", "e_y"]
            self.defaults = [9.81, 0.0, 0.1, 0.0, 0.0, 0.0]
        self.n_aux = len(self.aux_names)
        self.A, self.B, self.C = moment_coefficients(L)

    # index helpers: momentum component (direction d, moment k)
    def im(self, d, k):
        return 2 + d * self.nmom + k

    def pidx(self, name):
        return self.params.index(name)


def kp_hinv(h, eps):
    """Kurganov-Petrova regularised 1/h (reference Model.H:220)."""
    return sp.sqrt(2) * sp.Max(0, h) / sp.sqrt(h ** 4 + sp.Max(eps, h) ** 4)


def physical_flux(S, h, mom, hinv, g, d, pressure=True):
    """SME flux in direction d from the depth h, the momenta mom[dd][k] and an
    inverse depth hinv; every quadratic term is mom*mom*hinv (one 1/h factor,
    reference Model.H:53 / Numerics.H:55).  The model's own flux leaves out
    the hydrostatic pressure g h^2/2, which the reference keeps in the
    quasilinear matrix and the Riemann solver (Model.H:45-55, 75-92);
    pressure=True adds it.  Returns a list of length n_q."""
    L = S.L
    F = [sp.Integer(0)] * S.n_q
    F[1] = mom[d][0]
    for e in range(S.dim):  # row: momentum direction e
        val = mom[d][0] * mom[e][0] * hinv
        for j in range(1, L + 1):
            val += mom[d][j] * mom[e][j] * hinv / (2 * j + 1)
        if e == d and pressure:
            val += g * h ** 2 / 2
        F[S.im(e, 0)] = val
        for i in range(1, L + 1):
            val = (mom[d][0] * mom[e][i] + mom[e][0] * mom[d][i]) * hinv
            for j in range(1, L + 1):
                for k in range(1, L + 1):
                    a = S.A[i, j, k]
                    if a != 0:
                        val += a * mom[d][j] * mom[e][k] * hinv
            F[S.im(e, i)] = val
    return F


def ncp_matrix(S, h, mom, hinv, d):
    """Moment non-conservative matrix B_d (n_q x n_q): rows hu_i/hv_i (i>=1),
    columns hu_j (d = x) or hv_j (d = y), entry -u_e,m delta_ij + B_ijk u_e,k."""
    L = S.L
    M = sp.zeros(S.n_q, S.n_q)
    u = [[mom[dd][k] * hinv for k in range(S.nmom)] for dd in range(S.dim)]
    for e in range(S.dim):
        for i in range(1, L + 1):
            for j in range(1, L + 1):
                c = -u[e][0] if i == j else sp.Integer(0)
                for k in range(1, L + 1):
                    b = S.B[i, j, k]
                    if b != 0:
                        c += b * u[e][k]
                M[S.im(e, i), S.im(d, j)] = c
    return M


def moments(S, Q):
    return [[Q[S.im(d, k)] for k in range(S.nmom)] for d in range(S.dim)]


# --------------------------------------------------------------------------
# Model<T>
# --------------------------------------------------------------------------
def gen_model(S):
    nq, na, dim = S.n_q, S.n_aux, S.dim
    Q, Qa, p, n, X = arr("Q", nq), arr("Qaux", na), arr("p", len(S.params)), arr("n", dim), arr("X", 3)
    g = p[S.pidx("g")]
    h = Q[1]
    hinv = Qa[S.ihinv]
    mom = moments(S, Q)
    out = []
    w = out.append
    w("    static constexpr int n_dof_q    = %d;" % nq)
    w("    static constexpr int n_dof_qaux = %d;" % na)
    w("    static constexpr int n_parameters = %d;" % len(S.params))
    w("    static constexpr int dimension  = %d;" % dim)
    w("    static constexpr double dt_max = 5.0;")
    w("    static constexpr int n_dof_gradQ = 0;")
    w("    static constexpr bool has_diffusion = false;")
    w("    static constexpr bool has_free_surface = true;")
    w("    static constexpr int idx_b = 0;")
    w("    static constexpr int idx_h = 1;")
    w("    static constexpr int n_boundary_tags = 1;")
    w('    static const std::vector<std::string> get_boundary_tags() { return { "default" }; }')
    w("    static const std::vector<std::string> parameter_names() { return { %s }; }"
      % ", ".join('"%s"' % s for s in S.params))
    w("    static const std::vector<T> default_parameters() { return { %s }; }"
      % ", ".join(repr(float(v)) for v in S.defaults))

    def fn(name, args, exprs, size=None):
        w("    PORTABLE_FN static inline SimpleArray<T, %d> %s(" % (size or len(exprs), name))
        w(",\n".join("        " + a for a in args) + ")")
        w("    {")
        w(emit_body(exprs, size=size))
        w("    }")
        w("")

    qa3 = ["const T* Q", "const T* Qaux", "const T* p"]
    fluxes = []
    for d in range(dim):
        Fd = physical_flux(S, h, mom, hinv, g, d, pressure=False)
        fluxes.append(Fd)
        fn("flux_" + "xy"[d], qa3, Fd)
    NCs = []
    for d in range(dim):
        Bd = ncp_matrix(S, h, mom, hinv, d)
        # bathymetry column (row = mean momentum of direction d): g*h
        Bd[S.im(d, 0), 0] += g * h
        NCs.append(Bd)
        fn("nonconservative_matrix_" + "xy"[d], qa3, list(Bd))
    # eigenvalue bound in direction n (1/h regularised as max(1e-14, h),
    # reference Model.H:100-106)
    hreg = sp.Max(sp.Float(1e-14), h)
    u_n = sum(mom[d][0] * n[d] for d in range(dim)) / hreg
    c2 = g * sp.Max(0, h ** 5) / hreg ** 4
    for j in range(1, S.L + 1):
        a_n = sum(mom[d][j] * n[d] for d in range(dim)) / hreg
        c2 += sp.Rational(3, 2 * j + 1) * a_n ** 2
    c = sp.sqrt(c2)
    if dim == 1:   # 1-D: eigenvalues of n*A, i.e. n*(u -+ c) (Model.H:102-106)
        c = c * n[0]
    ev = [sp.Integer(0)] * nq
    ev[1] = u_n - c
    ev[2] = u_n + c
    for i in range(3, nq):
        ev[i] = u_n
    fn("eigenvalues", qa3 + ["const T* n"], ev)
    # source
    S_ = source_terms(S, Q, hinv, p)
    fn("source", qa3 + ["const T time", "const T dt", "const T* X"], S_)
    fn("flux", qa3, [e for Fd in fluxes for e in Fd])
    fn("nonconservative_matrix", qa3, [e for Bd in NCs for e in list(Bd)])
    # The reference's generator differentiates the source with hinv standing
    # for 1/h and prints 1/h back as hinv; its aux Jacobian is zero
    # (Model.H:155-193).  Same convention here.
    Hs = sp.Symbol("Hpos", positive=True)
    S_h = [sp.sympify(e).subs(hinv, 1 / Hs).subs(Q[1], Hs) for e in S_]
    J = []
    for i in range(nq):
        for j in range(nq):
            e = sp.diff(S_h[i], Hs if j == 1 else Q[j])
            e = e.replace(lambda x: x.is_Pow and x.base == Hs and x.exp.is_negative,
                          lambda x: hinv ** (-x.exp))
            J.append(e.subs(Hs, Q[1]))
    fn("source_jacobian_wrt_variables", qa3, J)
    fn("source_jacobian_wrt_aux_variables", qa3, [sp.Integer(0)] * (nq * na))
    # wet/dry momentum clamp
    t0 = 30 * sp.Max(0, h - sp.Rational(1, 100))
    uv = list(Q)
    for d in range(dim):
        for k in range(S.nmom):
            uv[S.im(d, k)] = sp.Max(-t0, sp.Min(Q[S.im(d, k)], t0))
    fn("update_variables", qa3 + ["const T dt"], uv)
    hinv_expr = kp_hinv(h, sp.Float(1e-8))
    ua = list(Qa)
    ua[S.ihinv] = hinv_expr
    fn("update_aux_variables", qa3 + ["const T time", "const T* X"], ua)
    Jua = [sp.diff(ua[k], Q[j]) if k == S.ihinv else sp.Integer(0) for k in range(na) for j in range(nq)]
    fn("update_aux_variables_jacobian_wrt_variables", qa3 + ["const T time", "const T* X"], Jua)
    # field-level overload filling the derivative aux slots ("d<var>d<axis>")
    # from whole fields through the solver's compute_derivative (the interface
    # of the reference's generated header, Model.H:250-262)
    deriv = []
    for k, nm in enumerate(S.aux_names):
        if nm.startswith("d") and len(nm) > 3 and nm[-2] == "d" and nm[-1] in "xyz":
            var, axis = nm[1:-2], nm[-1]
            qi = {"b": 0, "h": 1}.get(var)
            if qi is None and var.startswith("q"):
                qi = S.im(0, int(var[1:]))
            deriv.append((k, nm, qi, "xyz".index(axis)))
    if deriv:
        w("    static inline void update_aux_variables(")
        w("        T* const* Q,")
        w("        T* const* Qaux,")
        w("        const T dt,")
        w("        const ZoomyMesh& mesh)")
        w("    {")
        for k, nm, qi, ax in deriv:
            order = [0, 0, 0]
            order[ax] = 1
            w("    // Qaux[%d] (%s) = D^(%s) Q[%d]" % (k, nm, ",".join(str(o) for o in order[:S.dim]) + ("," if S.dim == 1 else ""), qi))
            w("    compute_derivative(Qaux[%d], Q[%d], %d, %d, %d, mesh);" % (k, qi, order[0], order[1], order[2]))
        w("    }")
        w("")
    ic = [sp.Integer(0)] * nq
    ic[0] = sp.Integer(1)
    fn("initial_condition", ["const T* X", "const T* p"], ic)
    # wall boundary condition: reflect the normal component of each pair
    bc = list(Q)
    for k in range(S.nmom):
        un = sum(Q[S.im(d, k)] * n[d] for d in range(dim))
        for d in range(dim):
            bc[S.im(d, k)] = Q[S.im(d, k)] - 2 * un * n[d]
    bcargs = ["const int bc_idx", "const T* Q", "const T* Qaux", "const T* p", "const T* n",
              "const T* X", "const T time", "const T dX"]
    for nm, vals, size in (("boundary_conditions", bc, nq), ("aux_boundary_conditions", list(Qa), na)):
        w("    PORTABLE_FN static inline SimpleArray<T, %d> %s(" % (size, nm))
        w(",\n".join("        " + a for a in bcargs) + ")")
        w("    {")
        w("    if (bc_idx == 0) {")
        w(emit_body(vals, size=size, indent="        "))
        w("    }")
        w("    SimpleArray<T, %d> default_res = {0};" % size)
        w("    return default_res;")
        w("    }")
        w("")
    return "\n".join(out)


def source_terms(S, Q, hinv, p):
    nq = S.n_q
    g = p[S.pidx("g")]
    mom = moments(S, Q)
    src = [sp.Integer(0)] * nq
    if S.variant == "malpasset":
        # reference Model.H:121 law: slope forcing minus linear slip friction
        rho, lam, ex = p[S.pidx("rho")], p[S.pidx("lambda_s")], p[S.pidx("e_x")]
        src[S.im(0, 0)] = ex * g * Q[1] - hinv * lam * Q[S.im(0, 0)] / rho
        return src
    nu, lam, nm = p[S.pidx("nu")], p[S.pidx("lambda")], p[S.pidx("n_manning")]
    ex, ey = p[S.pidx("e_x")], p[S.pidx("e_y")]
    e = [ex, ey]
    L = S.L
    # |u| regularised by 1e-24 (m/s)^2 so that the Jacobian term u^2/|u| is
    # finite at rest (0 * NaN would poison the Newton matrix even for n = 0)
    speed = sp.sqrt(sum((mom[d][0] * hinv) ** 2 for d in range(S.dim)) + sp.Float(1e-24))
    for d in range(S.dim):
        ub = sum(mom[d][k] for k in range(S.nmom)) * hinv  # bottom velocity
        for i in range(S.nmom):
            val = -(2 * i + 1) * (nu / lam) * ub
            for j in range(1, L + 1):
                if i >= 1 and S.C[i, j] != 0:
                    val += -(2 * i + 1) * nu * S.C[i, j] * mom[d][j] * hinv * hinv
            if i == 0:
                val += e[d] * g * Q[1]
                # Manning: -g n^2 u |u| h^(-1/3), with h^(-1/3) = cbrt(hinv)
                val += -g * nm ** 2 * (mom[d][0] * hinv) * speed * sp.cbrt(hinv)
            src[S.im(d, i)] = val
    return src


# --------------------------------------------------------------------------
# Numerics<T>
# --------------------------------------------------------------------------
def star_state(S, Q, bmax):
    """Hydrostatic reconstruction: h* = max(0, b + h - max(bL, bR)), momenta
    h* * u with u = hu / max(1e-14, h) (reference Numerics.H:40-47,67-80)."""
    hs_raw = Q[0] + Q[1] - bmax
    hs = sp.Max(0, hs_raw)
    hreg = sp.Max(sp.Float(1e-14), Q[1])
    mom = moments(S, Q)
    ms = [[mom[d][k] * hs / hreg for k in range(S.nmom)] for d in range(S.dim)]
    return hs_raw, hs, ms


def gen_numerics(S):
    nq, dim = S.n_q, S.dim
    QL, QR = arr("Q_minus", nq), arr("Q_plus", nq)
    p, n = arr("p", len(S.params)), arr("n", dim)
    g = p[S.pidx("g")]
    bmax = sp.Max(QL[0], QR[0])
    hsL_raw, hsL, msL = star_state(S, QL, bmax)
    hsR_raw, hsR, msR = star_state(S, QR, bmax)
    out = []
    w = out.append
    w("    static constexpr int n_dof_q = %d;" % nq)
    args6 = ["const T* Q_minus", "const T* Q_plus", "const T* Qaux_minus", "const T* Qaux_plus",
             "const T* p", "const T* n"]

    def fn(name, args, exprs):
        w("    PORTABLE_FN static inline SimpleArray<T, %d> %s(" % (len(exprs), name))
        w(",\n".join("        " + a for a in args) + ")")
        w("    {")
        w(emit_body(exprs))
        w("    }")
        w("")

    # central flux of the reconstructed states, 1/h* regularised (eps 1e-12)
    def Fn(hs_raw, hs, ms):
        hinv = sp.sqrt(2) * hs / sp.sqrt(hs ** 4 + sp.Max(sp.Float(1e-12), hs_raw) ** 4)
        tot = [sp.Integer(0)] * nq
        for d in range(dim):
            Fd = physical_flux(S, hs, ms, hinv, g, d)
            for i in range(nq):
                tot[i] += Fd[i] * n[d]
        return tot

    FL, FR = Fn(hsL_raw, hsL, msL), Fn(hsR_raw, hsR, msR)
    flux = [sp.Rational(1, 2) * (FL[i] + FR[i]) for i in range(nq)]
    fn("numerical_flux", args6, flux)

    # Rusanov speed (already halved, reference Numerics.H:81)
    def speeds(hs_raw, hs, ms):
        hreg = sp.Max(sp.Float(1e-14), hs_raw)
        un = sum(ms[d][0] * n[d] for d in range(dim)) / hreg
        c2 = g * hs ** 5 / hreg ** 4
        for j in range(1, S.L + 1):
            an = sum(ms[d][j] * n[d] for d in range(dim)) / hreg
            c2 += sp.Rational(3, 2 * j + 1) * an ** 2
        c = sp.sqrt(c2)
        return [sp.Abs(un + c), sp.Abs(un - c)]

    sL, sR = speeds(hsL_raw, hsL, msL), speeds(hsR_raw, hsR, msR)
    smax = sp.Rational(1, 2) * sp.Max(*(sL + sR))
    qsL = [sp.Integer(0), hsL] + [msL[d][k] for d in range(dim) for k in range(S.nmom)]
    qsR = [sp.Integer(0), hsR] + [msR[d][k] for d in range(dim) for k in range(S.nmom)]
    dq = [qsR[i] - qsL[i] for i in range(nq)]
    # midpoint of the reconstructed states for the non-conservative path integral
    hm = (hsL + hsR) / 2
    mm = [[(msL[d][k] + msR[d][k]) / 2 for k in range(S.nmom)] for d in range(dim)]
    hinv_m = kp_hinv(hm, sp.Float(1e-12)) if S.L >= 1 else None
    ncp = [sp.Integer(0)] * nq
    if S.L >= 1:
        Bn = sp.zeros(nq, nq)
        for d in range(dim):
            Bn += ncp_matrix(S, hm, mm, hinv_m, d) * n[d]
        for i in range(nq):
            ncp[i] = sp.Rational(1, 2) * sum(Bn[i, j] * dq[j] for j in range(nq) if Bn[i, j] != 0)
    right = [sp.Integer(0)] * nq
    left = [sp.Integer(0)] * nq
    for i in range(1, nq):
        right[i] = smax * dq[i] + ncp[i]
        left[i] = -smax * dq[i] + ncp[i]
    half_g = g / 2
    for d in range(dim):
        i0 = S.im(d, 0)
        right[i0] += n[d] * (-QR[1] ** 2 * half_g + half_g * hsR ** 2)
        left[i0] += n[d] * (QL[1] ** 2 * half_g - half_g * hsL ** 2)
    fn("numerical_fluctuations", args6, right + left)

    # w^T of the Jacobian of [numerical_flux, numerical_fluctuations] with
    # respect to both face states (the adjoint of a face; no counterpart in
    # the reference's headers, which the GPU adjoint differentiates with dual
    # numbers instead): g[0 .. nq) = d/dQ_minus, g[nq .. 2 nq) = d/dQ_plus.
    # The variant that mirrors the reference's shipped header goes without,
    # like that header.
    if S.variant != "malpasset":
        assert not any(str(s).startswith("Qaux") for e in flux + right + left for s in e.free_symbols)
        w("    PORTABLE_FN static inline void numerical_flux_fluct_vjp(")
        w(",\n".join("        " + a for a in args6 + ["const T* w", "T* g"]) + ")")
        w("    {")
        w(emit_vjp_body(flux + right + left, QL + QR))
        w("    }")
        w("")

    Q, Qa = arr("Q", nq), arr("Qaux", S.n_aux)
    hreg = sp.Max(sp.Float(1e-14), Q[1])
    mom = moments(S, Q)
    un = sum(mom[d][0] * n[d] for d in range(dim)) / hreg
    c2 = g * sp.Max(0, Q[1] ** 5) / hreg ** 4
    for j in range(1, S.L + 1):
        an = sum(mom[d][j] * n[d] for d in range(dim)) / hreg
        c2 += sp.Rational(3, 2 * j + 1) * an ** 2
    c = sp.sqrt(c2)
    fn("local_max_abs_eigenvalue", ["const T* Q", "const T* Qaux", "const T* p", "const T* n"],
       [sp.Max(sp.Abs(un + c), sp.Abs(un - c))])
    return "\n".join(out)


HEADER_PRE = """#pragma once
// Generated by models/gen_sme.py (%s). Do not edit by hand.
// Plugin interface of the reference's generated headers: Model<T> / Numerics<T>
// with static PORTABLE_FN members taking raw pointers and returning SimpleArray.
#include <cmath>
#include <array>

#ifndef ZOOMY_SIMPLE_ARRAY
#define ZOOMY_SIMPLE_ARRAY
template <typename T, int N>
struct SimpleArray {
    T data[N];
    T& operator[](int i) { return data[i]; }
    const T& operator[](int i) const { return data[i]; }
    T* begin() { return data; }
    const T* begin() const { return data; }
    T* end() { return data + N; }
    const T* end() const { return data + N; }
};
#endif

#include <vector>
#include <string>
#include <algorithm>

#ifdef __CUDACC__
#define PORTABLE_FN __host__ __device__
#else
#define PORTABLE_FN
#endif
"""


def write_model(S, outdir):
    d = os.path.join(outdir, S.name)
    os.makedirs(d, exist_ok=True)
    tag = "%s: dim=%d level=%d" % (S.name, S.dim, S.L)
    model = HEADER_PRE % tag + "\ntemplate <typename T>\nstruct Model {\n" + gen_model(S) + "\n};\n"
    num = (HEADER_PRE % tag + '#include "Model.H"\n\ntemplate <typename T>\nstruct Numerics {\n'
           + gen_numerics(S) + "\n};\n")
    with open(os.path.join(d, "Model.H"), "w") as f:
        f.write(model)
    with open(os.path.join(d, "Numerics.H"), "w") as f:
        f.write(num)
    return d


VARIANTS = {
    "sme1d_l0_malpasset": (1, 0, "malpasset"),
    "sme2d_l0": (2, 0, "sme"),
    "sme2d_l1": (2, 1, "sme"),
    "sme2d_l2": (2, 2, "sme"),
    "sme2d_l4": (2, 4, "sme"),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=HERE)
    ap.add_argument("names", nargs="*")
    a = ap.parse_args(argv)
    names = a.names or list(VARIANTS)
    for nm in names:
        dim, L, var = VARIANTS[nm]
        d = write_model(Spec(nm, dim, L, var), a.out)
        print("wrote", d)


if __name__ == "__main__":
    sys.exit(main())
