// Prelude that every translation unit includes before a generated model
// plugin (Model.H / Numerics.H).
//
// The generated headers define SimpleArray only if ZOOMY_SIMPLE_ARRAY is not
// yet defined (reference Model.H:5-17); their own definition is host-only.
// Predefining a __host__ __device__ SimpleArray here is what lets the same
// unmodified headers compile as device functions.  Heaviside is the one
// free function the generated bodies call by bare name (reference
// Model.H:242); sympy's convention Heaviside(0) = h0 is kept.
#pragma once
#include <cmath>
#include <array>
#include <vector>
#include <string>
#include <algorithm>
#include <type_traits>
#include <utility>

#ifdef __CUDACC__
#define ZSME_HD __host__ __device__
#else
#define ZSME_HD
#endif

#ifndef ZOOMY_SIMPLE_ARRAY
#define ZOOMY_SIMPLE_ARRAY
template <typename T, int N>
struct SimpleArray {
    T data[N];
    ZSME_HD T& operator[](int i) { return data[i]; }
    ZSME_HD const T& operator[](int i) const { return data[i]; }
    ZSME_HD T* begin() { return data; }
    ZSME_HD const T* begin() const { return data; }
    ZSME_HD T* end() { return data + N; }
    ZSME_HD const T* end() const { return data + N; }
};
#endif

// dual numbers and their std:: overloads, visible before the plugins are
// parsed (qualified std::sqrt etc. in a template bind at its definition)
#include "dual.h"

template <typename T>
ZSME_HD inline T Heaviside(T x, double h0) {
    return x < T(0) ? T(0) : (x > T(0) ? T(1) : T(h0));
}

// Mesh handle of the plugins' field-level update_aux_variables(Q, Qaux, dt,
// mesh) overload (reference UserFunctions.H:46-58), which fills derivative
// aux slots through compute_derivative(result, source, dx, dy, dz, mesh) on
// whole per-variable fields.  Here the handle carries the routine that
// serves each such request: the oracle computes the Green-Gauss derivative
// over its mesh (UserFunctions.H:60-112), the GPU library records which
// slot takes the derivative of which variable along which axis and runs a
// cell kernel for it.  Host only; instances on dual or counting scalars do
// not refresh (the derivative slots feed no step update).
struct ZoomyMesh {
    void (*derivative)(const ZoomyMesh& mesh, double* result, const double* source, int dx, int dy, int dz);
    void* ctx;
};
template <typename T>
inline void compute_derivative(T* result, const T* source, int dx, int dy, int dz, const ZoomyMesh& mesh) {
    if constexpr (std::is_same<T, double>::value) mesh.derivative(mesh, result, source, dx, dy, dz);
}

namespace zsme {

// The scalar type T of a plugin instantiation Model<T> (double, or a dual
// number for derivatives), so that the traits below detect the same
// functions whatever the scalar.
template <class M>
struct ScalarOf { using type = double; };
template <template <typename> class MT, typename T>
struct ScalarOf<MT<T>> { using type = T; };

// Trait detection mirroring the reference's SFINAE switches.
// update_variables(Q, Qaux, p, dt) present?  (TransportStep.hpp:22-29)
template <class M, typename = void>
struct HasUpdateVariables : std::false_type {};
template <class M>
struct HasUpdateVariables<M, std::void_t<decltype(M::update_variables(
    std::declval<const typename ScalarOf<M>::type*>(), std::declval<const typename ScalarOf<M>::type*>(),
    std::declval<const typename ScalarOf<M>::type*>(), std::declval<const typename ScalarOf<M>::type>()))>>
    : std::true_type {};

// Analytic dAux/dQ with the 3-argument signature?  (SourceStep.hpp:16-20)
// A 5-argument update_aux_variables_jacobian_wrt_variables does not match,
// exactly as in the reference, and the finite-difference path is taken.
template <class M, typename = void>
struct HasAuxJacobian : std::false_type {};
template <class M>
struct HasAuxJacobian<M, std::void_t<decltype(M::update_aux_variables_jacobian_wrt_variables(
    (const typename ScalarOf<M>::type*)nullptr, (const typename ScalarOf<M>::type*)nullptr,
    (const typename ScalarOf<M>::type*)nullptr))>> : std::true_type {};

// A generated numerical_flux_fluct_vjp(Q_minus, Q_plus, Qaux_minus,
// Qaux_plus, p, n, w, g): g = w^T d[numerical_flux, numerical_fluctuations]
// / d[Q_minus, Q_plus] in one reverse sweep.  Headers without it (the
// reference's own) are differentiated with dual numbers.
template <class N, typename = void>
struct HasFluxVJP : std::false_type {};
template <class N>
struct HasFluxVJP<N, std::void_t<decltype(N::numerical_flux_fluct_vjp(
    (const typename ScalarOf<N>::type*)nullptr, (const typename ScalarOf<N>::type*)nullptr,
    (const typename ScalarOf<N>::type*)nullptr, (const typename ScalarOf<N>::type*)nullptr,
    (const typename ScalarOf<N>::type*)nullptr, (const typename ScalarOf<N>::type*)nullptr,
    (const typename ScalarOf<N>::type*)nullptr, (typename ScalarOf<N>::type*)nullptr))>> : std::true_type {};

// Field-level update_aux_variables(T* const* Q, T* const* Qaux, T dt, const
// ZoomyMesh&) present?  (TransportStep.hpp:33-40: RefreshDerivativeAux runs
// only for plugins that emit it.)
template <class M, typename = void>
struct HasFieldAuxUpdate : std::false_type {};
template <class M>
struct HasFieldAuxUpdate<M, std::void_t<decltype(M::update_aux_variables(
    (typename ScalarOf<M>::type* const*)nullptr, (typename ScalarOf<M>::type* const*)nullptr,
    (typename ScalarOf<M>::type)0, std::declval<const ZoomyMesh&>()))>> : std::true_type {};

}  // namespace zsme
