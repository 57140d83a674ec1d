#pragma once
// Generated by models/gen_sme.py (sme2d_l1: dim=2 level=1). Do not edit by hand.
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
    static constexpr int n_dof_q    = 6;
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
    PORTABLE_FN static inline SimpleArray<T, 6> flux_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*((Q[2]*Q[2]) + 0.3333333333333333*(Q[3]*Q[3]));
    res[3] = 2.0*Q[2]*Q[3]*Qaux[0];
    res[4] = Qaux[0]*(Q[2]*Q[4] + 0.3333333333333333*Q[3]*Q[5]);
    res[5] = Qaux[0]*(Q[2]*Q[5] + Q[3]*Q[4]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> flux_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = Q[4];
    res[2] = Qaux[0]*(Q[2]*Q[4] + 0.3333333333333333*Q[3]*Q[5]);
    res[3] = Qaux[0]*(Q[2]*Q[5] + Q[3]*Q[4]);
    res[4] = Qaux[0]*((Q[4]*Q[4]) + 0.3333333333333333*(Q[5]*Q[5]));
    res[5] = 2.0*Q[4]*Q[5]*Qaux[0];
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 36> nonconservative_matrix_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 36> res;
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
    res[16] = 0.0;
    res[17] = 0.0;
    res[18] = 0.0;
    res[19] = 0.0;
    res[20] = 0.0;
    res[21] = (-Q[2]*Qaux[0]);
    res[22] = 0.0;
    res[23] = 0.0;
    res[24] = 0.0;
    res[25] = 0.0;
    res[26] = 0.0;
    res[27] = 0.0;
    res[28] = 0.0;
    res[29] = 0.0;
    res[30] = 0.0;
    res[31] = 0.0;
    res[32] = 0.0;
    res[33] = (-Q[4]*Qaux[0]);
    res[34] = 0.0;
    res[35] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 36> nonconservative_matrix_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 36> res;
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
    res[23] = (-Q[2]*Qaux[0]);
    res[24] = Q[1]*p[0];
    res[25] = 0.0;
    res[26] = 0.0;
    res[27] = 0.0;
    res[28] = 0.0;
    res[29] = 0.0;
    res[30] = 0.0;
    res[31] = 0.0;
    res[32] = 0.0;
    res[33] = 0.0;
    res[34] = 0.0;
    res[35] = (-Q[4]*Qaux[0]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> eigenvalues(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = std::max((T)1e-14, Q[1]);
    T t1 = (1.0/(t0));
    T t2 = std::sqrt((((Q[3]*n[0] + Q[5]*n[1])*(Q[3]*n[0] + Q[5]*n[1])) + (p[0]*std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1]))/(t0*t0))));
    T t3 = (Q[2]*n[0] + Q[4]*n[1]);
    T t4 = t1*t3;
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = t1*(t3 - t2);
    res[2] = t1*(t2 + t3);
    res[3] = t4;
    res[4] = t4;
    res[5] = t4;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> source(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T dt,
        const T* X)
    {
    T t0 = (1.0/(p[2]));
    T t1 = t0*(Q[2] + Q[3]);
    T t2 = Qaux[0]*p[1];
    T t3 = (Qaux[0]*Qaux[0]);
    T t4 = p[0]*(Qaux[0]*std::cbrt(Qaux[0]))*(p[3]*p[3])*std::sqrt((1e-24 + t3*(Q[2]*Q[2]) + t3*(Q[4]*Q[4])));
    T t5 = 4.0*Qaux[0];
    T t6 = 3.0*t2;
    T t7 = t0*(Q[4] + Q[5]);
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = ((-Q[2]*t4) - t1*t2 + Q[1]*p[0]*p[4]);
    res[3] = (-t6*(t1 + Q[3]*t5));
    res[4] = ((-Q[4]*t4) - t2*t7 + Q[1]*p[0]*p[5]);
    res[5] = (-t6*(t7 + Q[5]*t5));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> flux(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = 2.0*Qaux[0];
    T t1 = Qaux[0]*(Q[2]*Q[4] + 0.3333333333333333*Q[3]*Q[5]);
    T t2 = Qaux[0]*(Q[2]*Q[5] + Q[3]*Q[4]);
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*((Q[2]*Q[2]) + 0.3333333333333333*(Q[3]*Q[3]));
    res[3] = Q[2]*Q[3]*t0;
    res[4] = t1;
    res[5] = t2;
    res[6] = 0.0;
    res[7] = Q[4];
    res[8] = t1;
    res[9] = t2;
    res[10] = Qaux[0]*((Q[4]*Q[4]) + 0.3333333333333333*(Q[5]*Q[5]));
    res[11] = Q[4]*Q[5]*t0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 72> nonconservative_matrix(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = Q[1]*p[0];
    T t1 = (-Q[2]*Qaux[0]);
    T t2 = (-Q[4]*Qaux[0]);
    SimpleArray<T, 72> res;
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
    res[12] = t0;
    res[13] = 0.0;
    res[14] = 0.0;
    res[15] = 0.0;
    res[16] = 0.0;
    res[17] = 0.0;
    res[18] = 0.0;
    res[19] = 0.0;
    res[20] = 0.0;
    res[21] = t1;
    res[22] = 0.0;
    res[23] = 0.0;
    res[24] = 0.0;
    res[25] = 0.0;
    res[26] = 0.0;
    res[27] = 0.0;
    res[28] = 0.0;
    res[29] = 0.0;
    res[30] = 0.0;
    res[31] = 0.0;
    res[32] = 0.0;
    res[33] = t2;
    res[34] = 0.0;
    res[35] = 0.0;
    res[36] = 0.0;
    res[37] = 0.0;
    res[38] = 0.0;
    res[39] = 0.0;
    res[40] = 0.0;
    res[41] = 0.0;
    res[42] = 0.0;
    res[43] = 0.0;
    res[44] = 0.0;
    res[45] = 0.0;
    res[46] = 0.0;
    res[47] = 0.0;
    res[48] = 0.0;
    res[49] = 0.0;
    res[50] = 0.0;
    res[51] = 0.0;
    res[52] = 0.0;
    res[53] = 0.0;
    res[54] = 0.0;
    res[55] = 0.0;
    res[56] = 0.0;
    res[57] = 0.0;
    res[58] = 0.0;
    res[59] = t1;
    res[60] = t0;
    res[61] = 0.0;
    res[62] = 0.0;
    res[63] = 0.0;
    res[64] = 0.0;
    res[65] = 0.0;
    res[66] = 0.0;
    res[67] = 0.0;
    res[68] = 0.0;
    res[69] = 0.0;
    res[70] = 0.0;
    res[71] = t2;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 36> source_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (1.0/(p[2]));
    T t1 = t0*(Q[2] + Q[3]);
    T t2 = (Qaux[0]*Qaux[0]);
    T t3 = p[1]*t2;
    T t4 = (Q[2]*Q[2]);
    T t5 = (Q[4]*Q[4]);
    T t6 = std::sqrt((1e-24 + t2*t4 + t2*t5));
    T t7 = p[0]*(p[3]*p[3]);
    T t8 = t6*t7;
    T t9 = 1.3333333333333333*t8*(Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]));
    T t10 = (t7/(t6));
    T t11 = t10*(Qaux[0]*Qaux[0]*Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]))*(t4 + t5);
    T t12 = t10*(Qaux[0]*Qaux[0]*Qaux[0]*std::cbrt(Qaux[0]));
    T t13 = Qaux[0]*p[1];
    T t14 = t0*t13;
    T t15 = (t14 + t8*(Qaux[0]*std::cbrt(Qaux[0])));
    T t16 = (-t14);
    T t17 = (-Q[2]*Q[4]*t12);
    T t18 = 8.0*Qaux[0];
    T t19 = 3.0*t3;
    T t20 = (-3.0*t14);
    T t21 = (-3.0*t13*(t0 + 4.0*Qaux[0]));
    T t22 = t0*(Q[4] + Q[5]);
    SimpleArray<T, 36> res;
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
    res[12] = 0.0;
    res[13] = (Q[2]*t11 + Q[2]*t9 + p[0]*p[4] + t1*t3);
    res[14] = ((-t15) - t12*t4);
    res[15] = t16;
    res[16] = t17;
    res[17] = 0.0;
    res[18] = 0.0;
    res[19] = t19*(t1 + Q[3]*t18);
    res[20] = t20;
    res[21] = t21;
    res[22] = 0.0;
    res[23] = 0.0;
    res[24] = 0.0;
    res[25] = (Q[4]*t11 + Q[4]*t9 + p[0]*p[5] + t22*t3);
    res[26] = t17;
    res[27] = 0.0;
    res[28] = ((-t15) - t12*t5);
    res[29] = t16;
    res[30] = 0.0;
    res[31] = t19*(t22 + Q[5]*t18);
    res[32] = 0.0;
    res[33] = 0.0;
    res[34] = t20;
    res[35] = t21;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> source_jacobian_wrt_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> update_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T dt)
    {
    T t0 = 30.0*std::max((T)0.0, ((-1.0/100.0) + Q[1]));
    T t1 = (-t0);
    SimpleArray<T, 6> res;
    res[0] = Q[0];
    res[1] = Q[1];
    res[2] = std::max(t1, std::min(Q[2], t0));
    res[3] = std::max(t1, std::min(Q[3], t0));
    res[4] = std::max(t1, std::min(Q[4], t0));
    res[5] = std::max(t1, std::min(Q[5], t0));
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

    PORTABLE_FN static inline SimpleArray<T, 6> update_aux_variables_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    T t0 = std::max((T)1e-08, Q[1]);
    T t1 = ((Q[1]*Q[1]*Q[1]*Q[1]) + (t0*t0*t0*t0));
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = (std::sqrt(2.0)*((-(2.0*((Q[1]*Q[1]*Q[1]) + (t0*t0*t0)*Heaviside(((-1e-08) + Q[1]), (1.0/2.0)))*std::max((T)0.0, Q[1])/(t1))) + Heaviside(Q[1], (1.0/2.0)))/std::sqrt(t1));
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> initial_condition(
        const T* X,
        const T* p)
    {
    SimpleArray<T, 6> res;
    res[0] = 1.0;
    res[1] = 0.0;
    res[2] = 0.0;
    res[3] = 0.0;
    res[4] = 0.0;
    res[5] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> boundary_conditions(
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
        T t0 = (Q[2]*n[0] + Q[4]*n[1]);
        T t1 = 2.0*n[0];
        T t2 = (Q[3]*n[0] + Q[5]*n[1]);
        T t3 = 2.0*n[1];
        SimpleArray<T, 6> res;
        res[0] = Q[0];
        res[1] = Q[1];
        res[2] = (Q[2] - t0*t1);
        res[3] = (Q[3] - t1*t2);
        res[4] = (Q[4] - t0*t3);
        res[5] = (Q[5] - t2*t3);
        return res;
    }
    SimpleArray<T, 6> default_res = {0};
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
