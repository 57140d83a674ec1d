// Forward-mode dual numbers with N derivative directions, host and device.
//
// The generated model plugins are templates on their scalar type, so
// Model<Dual<N>> / Numerics<Dual<N>> evaluate a function and its Jacobian
// with respect to N seeded inputs in one pass; every comparison (max, min,
// fabs, the limiter and clamp branches) is decided by the values, so the
// derivative is that of the branch the primal evaluation takes.  The same
// header serves the GPU adjoint and the CPU tangent-linear check, so both use
// one convention at kinks: d|x| at x = 0 is +dx, and sqrt / cbrt have a zero
// derivative at exactly 0 (where they only appear multiplied by zero factors
// in the SME plugins: h*^(5/2) = h* h* sqrt(h*), ...).
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define ZD_HD __host__ __device__ __forceinline__
#else
#define ZD_HD inline
#endif

namespace zsme {

template <int N>
struct Dual {
    double v;
    double d[N];
    ZD_HD Dual() : v(0.0) {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    ZD_HD Dual(double x) : v(x) {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    ZD_HD static Dual seed(double x, int k) {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
    ZD_HD Dual& operator+=(const Dual& o) { v += o.v; for (int i = 0; i < N; ++i) d[i] += o.d[i]; return *this; }
    ZD_HD Dual& operator-=(const Dual& o) { v -= o.v; for (int i = 0; i < N; ++i) d[i] -= o.d[i]; return *this; }
    ZD_HD Dual& operator*=(const Dual& o) {
        for (int i = 0; i < N; ++i) d[i] = d[i] * o.v + v * o.d[i];
        v *= o.v;
        return *this;
    }
    ZD_HD Dual& operator/=(const Dual& o) {
        const double q = v / o.v;
        for (int i = 0; i < N; ++i) d[i] = (d[i] - q * o.d[i]) / o.v;
        v = q;
        return *this;
    }
};

template <int N> ZD_HD Dual<N> operator-(const Dual<N>& a) { Dual<N> r; r.v = -a.v; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }
template <int N> ZD_HD Dual<N> operator+(Dual<N> a, const Dual<N>& b) { return a += b; }
template <int N> ZD_HD Dual<N> operator-(Dual<N> a, const Dual<N>& b) { return a -= b; }
template <int N> ZD_HD Dual<N> operator*(Dual<N> a, const Dual<N>& b) { return a *= b; }
template <int N> ZD_HD Dual<N> operator/(Dual<N> a, const Dual<N>& b) { return a /= b; }
template <int N> ZD_HD Dual<N> operator+(Dual<N> a, double b) { a.v += b; return a; }
template <int N> ZD_HD Dual<N> operator+(double b, Dual<N> a) { a.v += b; return a; }
template <int N> ZD_HD Dual<N> operator-(Dual<N> a, double b) { a.v -= b; return a; }
template <int N> ZD_HD Dual<N> operator-(double b, const Dual<N>& a) { Dual<N> r = -a; r.v += b; return r; }
template <int N> ZD_HD Dual<N> operator*(Dual<N> a, double b) { a.v *= b; for (int i = 0; i < N; ++i) a.d[i] *= b; return a; }
template <int N> ZD_HD Dual<N> operator*(double b, Dual<N> a) { return a * b; }
template <int N> ZD_HD Dual<N> operator/(Dual<N> a, double b) { a.v /= b; for (int i = 0; i < N; ++i) a.d[i] /= b; return a; }
template <int N> ZD_HD Dual<N> operator/(double b, const Dual<N>& a) { return Dual<N>(b) / a; }

#define ZSME_DUAL_CMP(OP)                                                                        \
    template <int N> ZD_HD bool operator OP(const Dual<N>& a, const Dual<N>& b) { return a.v OP b.v; } \
    template <int N> ZD_HD bool operator OP(const Dual<N>& a, double b) { return a.v OP b; }          \
    template <int N> ZD_HD bool operator OP(double a, const Dual<N>& b) { return a OP b.v; }
ZSME_DUAL_CMP(<)
ZSME_DUAL_CMP(>)
ZSME_DUAL_CMP(<=)
ZSME_DUAL_CMP(>=)
ZSME_DUAL_CMP(==)
ZSME_DUAL_CMP(!=)
#undef ZSME_DUAL_CMP

template <int N> ZD_HD double value(const Dual<N>& a) { return a.v; }
ZD_HD double value(double a) { return a; }

template <int N> ZD_HD Dual<N> dual_sqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = ::sqrt(a.v);
    const double s = r.v > 0.0 ? 0.5 / r.v : 0.0;
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
template <int N> ZD_HD Dual<N> dual_cbrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = ::cbrt(a.v);
    const double s = r.v != 0.0 ? 1.0 / (3.0 * r.v * r.v) : 0.0;
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
template <int N> ZD_HD Dual<N> dual_fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }

}  // namespace zsme

// The generated plugins call std::sqrt / std::fabs / std::cbrt / std::abs
// qualified; std::max / std::min work through operator<.
namespace std {
template <int N> ZD_HD zsme::Dual<N> sqrt(const zsme::Dual<N>& a) { return zsme::dual_sqrt(a); }
template <int N> ZD_HD zsme::Dual<N> cbrt(const zsme::Dual<N>& a) { return zsme::dual_cbrt(a); }
template <int N> ZD_HD zsme::Dual<N> fabs(const zsme::Dual<N>& a) { return zsme::dual_fabs(a); }
template <int N> ZD_HD zsme::Dual<N> abs(const zsme::Dual<N>& a) { return zsme::dual_fabs(a); }
template <int N> ZD_HD bool isfinite(const zsme::Dual<N>& a) { return isfinite(a.v); }
// x^e for a constant exponent (zero derivative at x = 0, as for sqrt)
template <int N> ZD_HD zsme::Dual<N> pow(const zsme::Dual<N>& a, double e) {
    zsme::Dual<N> r;
    r.v = pow(a.v, e);
    const double s = a.v != 0.0 ? e * pow(a.v, e - 1.0) : 0.0;
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
}  // namespace std
