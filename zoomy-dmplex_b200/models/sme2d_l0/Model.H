#pragma once
// Generated by models/gen_sme.py (sme2d_l0: dim=2 level=0). Do not edit by hand.
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
    static constexpr int n_dof_q    = 4;
    static constexpr int n_dof_qaux = 1;
    static constexpr int n_parameters = 6;
    static constexpr int dimension  = 2;
    static constexpr double dt_max = 5.0;
    static constexpr int n_dof_gradQ = 0;
    static constexpr bool has_diffusion = false;
    static constexpr bool has_free_surface = true;
    static constexpr int idx_b = 0;
    static constexpr int idx_h = 1;
    static constexpr int n_boundary_tags = 1;
    static const std::vector<std::string> get_boundary_tags() { return { "default" }; }
    static const std::vector<std::string> parameter_names() { return { "g", "nu", "lambda", "n_manning", "e_x", "e_y" }; }
    static const std::vector<T> default_parameters() { return { 9.81, 0.0, 0.1, 0.0, 0.0, 0.0 }; }
    PORTABLE_FN static inline SimpleArray<T, 4> flux_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*(Q[2]*Q[2]);
    res[3] = Q[2]*Q[3]*Qaux[0];
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> flux_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = Q[3];
    res[2] = Q[2]*Q[3]*Qaux[0];
    res[3] = Qaux[0]*(Q[3]*Q[3]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 16> nonconservative_matrix_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 16> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = 0.0;
    res[8] = Q[1]*p[0];
    res[9] = 0.0;
    res[10] = 0.0;
    res[11] = 0.0;
    res[12] = 0.0;
    res[13] = 0.0;
    res[14] = 0.0;
    res[15] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 16> nonconservative_matrix_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 16> res;
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
    res[12] = Q[1]*p[0];
    res[13] = 0.0;
    res[14] = 0.0;
    res[15] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> eigenvalues(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = (1.0/(std::max((T)1e-14, Q[1])));
    T t1 = t0*std::sqrt(p[0])*std::sqrt(std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1])));
    T t2 = (Q[2]*n[0] + Q[3]*n[1]);
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = t0*(t2 - t1);
    res[2] = t0*(t1 + t2);
    res[3] = t0*t2;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> source(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T dt,
        const T* X)
    {
    T t0 = (Qaux[0]*p[1]/(p[2]));
    T t1 = (Qaux[0]*Qaux[0]);
    T t2 = p[0]*(Qaux[0]*std::cbrt(Qaux[0]))*(p[3]*p[3])*std::sqrt((1e-24 + t1*(Q[2]*Q[2]) + t1*(Q[3]*Q[3])));
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = ((-Q[2]*t0) - Q[2]*t2 + Q[1]*p[0]*p[4]);
    res[3] = ((-Q[3]*t0) - Q[3]*t2 + Q[1]*p[0]*p[5]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 8> flux(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = Q[2]*Q[3]*Qaux[0];
    SimpleArray<T, 8> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*(Q[2]*Q[2]);
    res[3] = t0;
    res[4] = 0.0;
    res[5] = Q[3];
    res[6] = t0;
    res[7] = Qaux[0]*(Q[3]*Q[3]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 32> nonconservative_matrix(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = Q[1]*p[0];
    SimpleArray<T, 32> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = 0.0;
    res[8] = t0;
    res[9] = 0.0;
    res[10] = 0.0;
    res[11] = 0.0;
    res[12] = 0.0;
    res[13] = 0.0;
    res[14] = 0.0;
    res[15] = 0.0;
    res[16] = 0.0;
    res[17] = 0.0;
    res[18] = 0.0;
    res[19] = 0.0;
    res[20] = 0.0;
    res[21] = 0.0;
    res[22] = 0.0;
    res[23] = 0.0;
    res[24] = 0.0;
    res[25] = 0.0;
    res[26] = 0.0;
    res[27] = 0.0;
    res[28] = t0;
    res[29] = 0.0;
    res[30] = 0.0;
    res[31] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 16> source_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (Qaux[0]*Qaux[0]);
    T t1 = (p[1]/(p[2]));
    T t2 = t0*t1;
    T t3 = (Q[2]*Q[2]);
    T t4 = (Q[3]*Q[3]);
    T t5 = std::sqrt((1e-24 + t0*t3 + t0*t4));
    T t6 = p[0]*(p[3]*p[3]);
    T t7 = t5*t6;
    T t8 = 1.3333333333333333*t7*(Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]));
    T t9 = (t6/(t5));
    T t10 = t9*(Qaux[0]*Qaux[0]*Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]))*(t3 + t4);
    T t11 = t9*(Qaux[0]*Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]));
    T t12 = (Qaux[0]*t1 + t7*(Qaux[0]*std::cbrt(Qaux[0])));
    T t13 = (-Q[2]*Q[3]*t11);
    SimpleArray<T, 16> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    res[6] = 0.0;
    res[7] = 0.0;
    res[8] = 0.0;
    res[9] = (Q[2]*t10 + Q[2]*t2 + Q[2]*t8 + p[0]*p[4]);
    res[10] = ((-t12) - t11*t3);
    res[11] = t13;
    res[12] = 0.0;
    res[13] = (Q[3]*t10 + Q[3]*t2 + Q[3]*t8 + p[0]*p[5]);
    res[14] = t13;
    res[15] = ((-t12) - t11*t4);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> source_jacobian_wrt_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> update_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T dt)
    {
    T t0 = 30.0*std::max((T)0.0, ((-1.0/100.0) + Q[1]));
    T t1 = (-t0);
    SimpleArray<T, 4> res;
    res[0] = Q[0];
    res[1] = Q[1];
    res[2] = std::max(t1, std::min(Q[2], t0));
    res[3] = std::max(t1, std::min(Q[3], t0));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 1> update_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    SimpleArray<T, 1> res;
    res[0] = (std::sqrt(2.0)*std::max((T)0.0, Q[1])/std::sqrt(((Q[1]*Q[1]*Q[1]*Q[1]) + (std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])*std::max((T)1e-08, Q[1])))));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> update_aux_variables_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    T t0 = std::max((T)1e-08, Q[1]);
    T t1 = ((Q[1]*Q[1]*Q[1]*Q[1]) + (t0*t0*t0*t0));
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = (std::sqrt(2.0)*((-(2.0*((Q[1]*Q[1]*Q[1]) + (t0*t0*t0)*Heaviside(((-1e-08) + Q[1]), (1.0/2.0)))*std::max((T)0.0, Q[1])/(t1))) + Heaviside(Q[1], (1.0/2.0)))/std::sqrt(t1));
    res[2] = 0.0;
    res[3] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> initial_condition(
        const T* X,
        const T* p)
    {
    SimpleArray<T, 4> res;
    res[0] = 1.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 4> boundary_conditions(
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
        T t0 = (2.0*Q[2]*n[0] + 2.0*Q[3]*n[1]);
        SimpleArray<T, 4> res;
        res[0] = Q[0];
        res[1] = Q[1];
        res[2] = (Q[2] - n[0]*t0);
        res[3] = (Q[3] - n[1]*t0);
        return res;
    }
    SimpleArray<T, 4> default_res = {0};
    return default_res;
    }

    PORTABLE_FN static inline SimpleArray<T, 1> aux_boundary_conditions(
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
        SimpleArray<T, 1> res;
        res[0] = Qaux[0];
        return res;
    }
    SimpleArray<T, 1> default_res = {0};
    return default_res;
    }

};
