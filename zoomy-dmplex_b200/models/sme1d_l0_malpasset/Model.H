#pragma once
// Generated by models/gen_sme.py (sme1d_l0_malpasset: dim=1 level=0). Do not edit by hand.
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

template <typename T>
struct Model {
    static constexpr int n_dof_q    = 3;
    static constexpr int n_dof_qaux = 4;
    static constexpr int n_parameters = 5;
    static constexpr int dimension  = 1;
    static constexpr double dt_max = 5.0;
    static constexpr int n_dof_gradQ = 0;
    static constexpr bool has_diffusion = false;
    static constexpr bool has_free_surface = true;
    static constexpr int idx_b = 0;
    static constexpr int idx_h = 1;
    static constexpr int n_boundary_tags = 1;
    static const std::vector<std::string> get_boundary_tags() { return { "default" }; }
    static const std::vector<std::string> parameter_names() { return { "g", "rho", "nu", "lambda_s", "e_x" }; }
    static const std::vector<T> default_parameters() { return { 9.81, 1.0, 1.0, 0.5, 0.0 }; }
    PORTABLE_FN static inline SimpleArray<T, 3> flux_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 3> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[3]*(Q[2]*Q[2]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 9> nonconservative_matrix_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 9> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = Q[1]*p[0];
    res[7] = 0.0;
    res[8] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 3> eigenvalues(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = (1.0/(std::max((T)1e-14, Q[1])));
    T t1 = t0*std::sqrt(p[0])*std::sqrt(std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1])));
    T t2 = n[0]*t0;
    SimpleArray<T, 3> res;
    res[0] = 0.0;
    res[1] = t2*(Q[2] - t1);
    res[2] = t2*(Q[2] + t1);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 3> source(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T dt,
        const T* X)
    {
    SimpleArray<T, 3> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = (Q[1]*p[0]*p[4] - (Q[2]*Qaux[3]*p[3]/(p[1])));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 3> flux(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 3> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[3]*(Q[2]*Q[2]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 9> nonconservative_matrix(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 9> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = Q[1]*p[0];
    res[7] = 0.0;
    res[8] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 9> source_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (p[3]/(p[1]));
    SimpleArray<T, 9> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = (p[0]*p[4] + Q[2]*t0*(Qaux[3]*Qaux[3]));
    res[8] = (-Qaux[3]*t0);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> source_jacobian_wrt_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = 0.0;
    res[8] = 0.0;
    res[9] = 0.0;
    res[10] = 0.0;
    res[11] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 3> update_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T dt)
    {
    T t0 = 30.0*std::max((T)0.0, ((-1.0/100.0) + Q[1]));
    SimpleArray<T, 3> res;
    res[0] = Q[0];
    res[1] = Q[1];
    res[2] = std::max((-t0), std::min(Q[2], t0));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> update_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    SimpleArray<T, 4> res;
    res[0] = Qaux[0];
    res[1] = Qaux[1];
    res[2] = Qaux[2];
    res[3] = (std::sqrt(2.0)*std::max((T)0.0, Q[1])/std::sqrt(((Q[1]*Q[1]*Q[1]*Q[1]) + (std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])))));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> update_aux_variables_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    T t0 = std::max((T)1e-08, Q[1]);
    T t1 = ((Q[1]*Q[1]*Q[1]*Q[1]) + (t0*t0*t0*t0));
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = 0.0;
    res[8] = 0.0;
    res[9] = 0.0;
    res[10] = (std::sqrt(2.0)*((-(2.0*((Q[1]*Q[1]*Q[1]) + (t0*t0*t0)*Heaviside(((-1e-08) + Q[1]), (1.0/2.0)))*std::max((T)0.0, Q[1])/(t1))) + Heaviside(Q[1], (1.0/2.0)))/std::sqrt(t1));
    res[11] = 0.0;
    return res;
    }

    static inline void update_aux_variables(
        T* const* Q,
        T* const* Qaux,
        const T dt,
        const ZoomyMesh& mesh)
    {
    // Qaux[0] (dq0dx) = D^(1,) Q[2]
    compute_derivative(Qaux[0], Q[2], 1, 0, 0, mesh);
    // Qaux[1] (dhdx) = D^(1,) Q[1]
    compute_derivative(Qaux[1], Q[1], 1, 0, 0, mesh);
    // Qaux[2] (dbdx) = D^(1,) Q[0]
    compute_derivative(Qaux[2], Q[0], 1, 0, 0, mesh);
    }

    PORTABLE_FN static inline SimpleArray<T, 3> initial_condition(
        const T* X,
        const T* p)
    {
    SimpleArray<T, 3> res;
    res[0] = 1.0;
    res[1] = 0.0;
    res[2] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 3> boundary_conditions(
        const int bc_idx,
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n,
        const T* X,
        const T time,
        const T dX)
    {
    if (bc_idx == 0) {
        SimpleArray<T, 3> res;
        res[0] = Q[0];
        res[1] = Q[1];
        res[2] = Q[2]*(1.0 - 2.0*(n[0]*n[0]));
        return res;
    }
    SimpleArray<T, 3> default_res = {0};
    return default_res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> aux_boundary_conditions(
        const int bc_idx,
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n,
        const T* X,
        const T time,
        const T dX)
    {
    if (bc_idx == 0) {
        SimpleArray<T, 4> res;
        res[0] = Qaux[0];
        res[1] = Qaux[1];
        res[2] = Qaux[2];
        res[3] = Qaux[3];
        return res;
    }
    SimpleArray<T, 4> default_res = {0};
    return default_res;
    }

};
