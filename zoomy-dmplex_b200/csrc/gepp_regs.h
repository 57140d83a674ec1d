// The two Gaussian eliminations with partial pivoting of the implicit
// source step, SourceStep::SolveLinearSystem (SourceStep.hpp:211-242): on a
// register block (the Newton fast path) and on the full matrix in local
// memory (the generic path).  Host and device: the host build is what the
// CPU test of the register form compiles (tests/gepp_regs_check.cpp).
#pragma once
#include <cmath>
#include <cstring>

#ifdef __CUDACC__
#define ZSME_GEPP_INLINE __host__ __device__ __forceinline__
#define ZSME_GEPP_FN __host__ __device__
#else
#define ZSME_GEPP_INLINE inline
#define ZSME_GEPP_FN inline
#endif

namespace zsme {

// c ? a : b as a bitwise blend.  The row swaps below are written with it
// because the compiler turns a chain of plain selects (or of predicated
// swaps) on the pivot row index into a dynamically indexed local-memory
// array once the block is 5 x 5 (240 bytes of stack); the blend keeps the
// block in registers and moves the same bits.
ZSME_GEPP_INLINE double blend(bool c, double a, double b) {
    const long long m = -(long long)c;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((__double_as_longlong(a) & m) | (__double_as_longlong(b) & ~m));
#else
    long long ia, ib;
    std::memcpy(&ia, &a, sizeof ia);
    std::memcpy(&ib, &b, sizeof ib);
    const long long r = (ia & m) | (ib & ~m);
    double o;
    std::memcpy(&o, &r, sizeof o);
    return o;
#endif
}

// GEPP of SolveLinearSystem on an NB x NB block held in registers (all
// indices compile-time; row swaps are bitwise blends).  Returns false on a
// pivot below 1e-14.
template <int NB>
ZSME_GEPP_INLINE bool gepp_regs(double (&A)[NB][NB], double (&b)[NB], double (&x)[NB]) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        int mr = k;
        double mv = fabs(A[k][k]);
#pragma unroll
        for (int i = k + 1; i < NB; ++i) {
            const double v = fabs(A[i][k]);
            if (v > mv) { mv = v; mr = i; }
        }
        if (mv < 1e-14) ok = false;
        // swap rows k and mr of [A | b] (columns k.. of A)
#pragma unroll
        for (int j = k; j <= NB; ++j) {
            const double pk = j < NB ? A[k][j] : b[k];
            double piv = pk;
#pragma unroll
            for (int i = k + 1; i < NB; ++i) {
                const double ai = j < NB ? A[i][j] : b[i];
                const double ni = blend(mr == i, pk, ai);
                piv = blend(mr == i, ai, piv);
                if (j < NB) A[i][j] = ni;
                else b[i] = ni;
            }
            if (j < NB) A[k][j] = piv;
            else b[k] = piv;
        }
        const double pkk = A[k][k];
        const double bk = b[k];
#pragma unroll
        for (int i = k + 1; i < NB; ++i) {
            const double fct = A[i][k] / pkk;
#pragma unroll
            for (int j = k; j < NB; ++j) A[i][j] -= fct * A[k][j];
            b[i] -= fct * bk;
        }
    }
#pragma unroll
    for (int i = NB - 1; i >= 0; --i) {
        double sum = 0.0;
#pragma unroll
        for (int j = i + 1; j < NB; ++j) sum += A[i][j] * x[j];
        x[i] = (b[i] - sum) / A[i][i];
    }
    return ok;
}

// Generic GEPP over the full matrix (local memory).
template <int NQ>
ZSME_GEPP_FN bool gepp_full(double* J, double* bv, double* xv) {
    for (int k = 0; k < NQ; ++k) {
        int mr = k;
        double mv = fabs(J[k * NQ + k]);
        for (int i = k + 1; i < NQ; ++i)
            if (fabs(J[i * NQ + k]) > mv) { mv = fabs(J[i * NQ + k]); mr = i; }
        if (mv < 1e-14) return false;
        if (mr != k) {
            for (int j = k; j < NQ; ++j) { const double tt = J[k * NQ + j]; J[k * NQ + j] = J[mr * NQ + j]; J[mr * NQ + j] = tt; }
            const double tt = bv[k]; bv[k] = bv[mr]; bv[mr] = tt;
        }
        for (int i = k + 1; i < NQ; ++i) {
            const double fct = J[i * NQ + k] / J[k * NQ + k];
            for (int j = k; j < NQ; ++j) J[i * NQ + j] -= fct * J[k * NQ + j];
            bv[i] -= fct * bv[k];
        }
    }
    for (int i = NQ - 1; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1; j < NQ; ++j) sum += J[i * NQ + j] * xv[j];
        xv[i] = (bv[i] - sum) / J[i * NQ + i];
    }
    return true;
}

}  // namespace zsme
