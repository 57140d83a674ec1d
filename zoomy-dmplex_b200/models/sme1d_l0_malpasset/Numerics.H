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
#include "Model.H"

template <typename T>
struct Numerics {
    static constexpr int n_dof_q = 3;
    PORTABLE_FN static inline SimpleArray<T, 3> numerical_flux(
        const T* Q_minus,
        const T* Q_plus,
        const T* Qaux_minus,
        const T* Qaux_plus,
        const T* p,
        const T* n)
    {
    T t0 = std::max((T)1e-14, Q_minus[1]);
    T t1 = (-std::max(Q_minus[0], Q_plus[0]));
    T t2 = (Q_minus[0] + Q_minus[1] + t1);
    T t3 = std::max((T)0.0, t2);
    T t4 = std::max((T)1e-14, Q_plus[1]);
    T t5 = (Q_plus[0] + Q_plus[1] + t1);
    T t6 = std::max((T)0.0, t5);
    T t7 = 2.0*std::sqrt(2.0);
    SimpleArray<T, 3> res;
    res[0] = 0.0;
    res[1] = 0.5*n[0]*((Q_minus[2]*t3/(t0)) + (Q_plus[2]*t6/(t4)));
    res[2] = 0.25*n[0]*((t3*t3)*(p[0] + (t3*t7*(Q_minus[2]*Q_minus[2])/((t0*t0)*std::sqrt(((t3*t3*t3*t3) + (std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2))))))) + (t6*t6)*(p[0] + (t6*t7*(Q_plus[2]*Q_plus[2])/((t4*t4)*std::sqrt(((t6*t6*t6*t6) + (std::max((T)1e-12, t5)*std::max((T)1e-12, t5)*std::max((T)1e-12, t5)*std::max((T)1e-12, t5))))))));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 6> numerical_fluctuations(
        const T* Q_minus,
        const T* Q_plus,
        const T* Qaux_minus,
        const T* Qaux_plus,
        const T* p,
        const T* n)
    {
    T t0 = (-std::max(Q_minus[0], Q_plus[0]));
    T t1 = (Q_minus[0] + Q_minus[1] + t0);
    T t2 = std::max((T)0.0, t1);
    T t3 = (Q_plus[0] + Q_plus[1] + t0);
    T t4 = std::max((T)0.0, t3);
    T t5 = (1.0/(std::max((T)1e-14, t1)));
    T t6 = (Q_minus[2]*t2/(std::max((T)1e-14, Q_minus[1])));
    T t7 = n[0]*t6;
    T t8 = std::sqrt(p[0]);
    T t9 = t5*t8*(t2*t2*std::sqrt(t2));
    T t10 = (1.0/(std::max((T)1e-14, t3)));
    T t11 = (Q_plus[2]*t4/(std::max((T)1e-14, Q_plus[1])));
    T t12 = n[0]*t11;
    T t13 = t10*t8*(t4*t4*std::sqrt(t4));
    T t14 = std::max(t10*std::fabs((t12 + t13)), std::max(t5*std::fabs((t7 + t9)), std::max(t10*std::fabs((t12 - t13)), t5*std::fabs((t7 - t9)))));
    T t15 = 0.5*t14*(t2 - t4);
    T t16 = n[0]*p[0];
    T t17 = t14*(t6 - t11);
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = (-t15);
    res[2] = ((-0.5*t17) - 0.5*t16*((Q_plus[1]*Q_plus[1]) - (t4*t4)));
    res[3] = 0.0;
    res[4] = t15;
    res[5] = (0.5*t17 + 0.5*t16*((Q_minus[1]*Q_minus[1]) - (t2*t2)));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 1> local_max_abs_eigenvalue(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = (1.0/(std::max((T)1e-14, Q[1])));
    T t1 = Q[2]*n[0];
    T t2 = t0*std::sqrt(p[0])*std::sqrt(std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1])));
    SimpleArray<T, 1> res;
    res[0] = std::max(t0*std::fabs((t1 + t2)), t0*std::fabs((t1 - t2)));
    return res;
    }

};
