// FLOP COUNTING -- test infrastructure, not the product.
//
// A scalar type for the oracle that behaves as a double and counts every
// floating-point operation done on state or parameter values: the oracle
// instantiated on it (Oracle<MT, NT, Counted>) counts the algorithmic FP64
// operations of the reference's step.  Geometry (double in the oracle) is
// precomputed data and not counted; comparisons, min / max, fabs and sign
// changes are selects, not arithmetic, and not counted either.
//
// Counts are kept per phase of the step, named after the step's kernels:
//   PREP    stage constraints, neighbour bounds, gradient, limiting,
//           reconstruction of the face states
//   FACE    face aux, numerical flux and fluctuations, boundary ghost
//           states, the area products
//   GATHER  the per-cell sums of the face contributions, / volume, the SSP
//           stage combination
//   FINAL   step constraints, implicit Newton source, CFL dt
// The counters are plain globals: count with one oracle thread.
#pragma once
#include <cmath>

namespace zsme_flops {
enum Op { ADD, MUL, DIV, SQRT, OTHER, NOPS };   // ADD: + and -; OTHER: cbrt, pow
enum Phase { PREP, FACE, GATHER, FINAL, NPH };
inline long long counts[NPH][NOPS];
inline int phase = FINAL;
inline void tick(int op) { ++counts[phase][op]; }
}  // namespace zsme_flops

namespace zsme {

struct Counted {
    double v;
    Counted() : v(0.0) {}
    Counted(double x) : v(x) {}
    Counted& operator+=(const Counted& o) { zsme_flops::tick(zsme_flops::ADD); v += o.v; return *this; }
    Counted& operator-=(const Counted& o) { zsme_flops::tick(zsme_flops::ADD); v -= o.v; return *this; }
    Counted& operator*=(const Counted& o) { zsme_flops::tick(zsme_flops::MUL); v *= o.v; return *this; }
    Counted& operator/=(const Counted& o) { zsme_flops::tick(zsme_flops::DIV); v /= o.v; return *this; }
};

inline Counted operator-(const Counted& a) { return Counted(-a.v); }
inline Counted operator+(Counted a, const Counted& b) { return a += b; }
inline Counted operator-(Counted a, const Counted& b) { return a -= b; }
inline Counted operator*(Counted a, const Counted& b) { return a *= b; }
inline Counted operator/(Counted a, const Counted& b) { return a /= b; }
inline Counted operator+(Counted a, double b) { return a += Counted(b); }
inline Counted operator+(double b, Counted a) { return Counted(b) += a; }
inline Counted operator-(Counted a, double b) { return a -= Counted(b); }
inline Counted operator-(double b, const Counted& a) { return Counted(b) -= a; }
inline Counted operator*(Counted a, double b) { return a *= Counted(b); }
inline Counted operator*(double b, Counted a) { return Counted(b) *= a; }
inline Counted operator/(Counted a, double b) { return a /= Counted(b); }
inline Counted operator/(double b, const Counted& a) { return Counted(b) /= a; }

#define ZSME_COUNTED_CMP(OP)                                                             \
    inline bool operator OP(const Counted& a, const Counted& b) { return a.v OP b.v; } \
    inline bool operator OP(const Counted& a, double b) { return a.v OP b; }          \
    inline bool operator OP(double a, const Counted& b) { return a OP b.v; }
ZSME_COUNTED_CMP(<)
ZSME_COUNTED_CMP(>)
ZSME_COUNTED_CMP(<=)
ZSME_COUNTED_CMP(>=)
ZSME_COUNTED_CMP(==)
ZSME_COUNTED_CMP(!=)
#undef ZSME_COUNTED_CMP

inline double value(const Counted& a) { return a.v; }

}  // namespace zsme

// The generated plugins call std::sqrt / std::fabs / std::cbrt / std::abs /
// std::pow qualified; std::max / std::min work through operator<.
namespace std {
inline zsme::Counted sqrt(const zsme::Counted& a) { zsme_flops::tick(zsme_flops::SQRT); return zsme::Counted(::sqrt(a.v)); }
inline zsme::Counted cbrt(const zsme::Counted& a) { zsme_flops::tick(zsme_flops::OTHER); return zsme::Counted(::cbrt(a.v)); }
inline zsme::Counted fabs(const zsme::Counted& a) { return zsme::Counted(::fabs(a.v)); }
inline zsme::Counted abs(const zsme::Counted& a) { return zsme::Counted(::fabs(a.v)); }
inline bool isfinite(const zsme::Counted& a) { return isfinite(a.v); }
inline zsme::Counted pow(const zsme::Counted& a, double e) { zsme_flops::tick(zsme_flops::OTHER); return zsme::Counted(::pow(a.v, e)); }
}  // namespace std
