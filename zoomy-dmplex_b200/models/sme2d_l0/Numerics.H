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
#include "Model.H"

template <typename T>
struct Numerics {
    static constexpr int n_dof_q = 4;
    PORTABLE_FN static inline SimpleArray<T, 4> numerical_flux(
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
    T t4 = (t3/(t0));
    T t5 = Q_minus[2]*n[0];
    T t6 = Q_minus[3]*n[1];
    T t7 = std::max((T)1e-14, Q_plus[1]);
    T t8 = (Q_plus[0] + Q_plus[1] + t1);
    T t9 = std::max((T)0.0, t8);
    T t10 = (t9/(t7));
    T t11 = Q_plus[2]*n[0];
    T t12 = Q_plus[3]*n[1];
    T t13 = std::sqrt(2.0);
    T t14 = (1.0/((t0*t0)*std::sqrt(((t3*t3*t3*t3) + (std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2))))));
    T t15 = t13*t14*(t3*t3*t3);
    T t16 = (1.0/((t7*t7)*std::sqrt(((t9*t9*t9*t9) + (std::max((T)1e-12, t8)*std::max((T)1e-12, t8)*std::max((T)1e-12, t8)*std::max((T)1e-12, t8))))));
    T t17 = t13*t16*(t9*t9*t9);
    T t18 = (t3*t3);
    T t19 = 2.0*t13;
    T t20 = t14*t19*t3;
    T t21 = 0.5*n[0];
    T t22 = (t9*t9);
    T t23 = t16*t19*t9;
    T t24 = 0.5*n[1];
    SimpleArray<T, 4> res;
    res[0] = 0.0;
    res[1] = (0.5*t10*t11 + 0.5*t10*t12 + 0.5*t4*t5 + 0.5*t4*t6);
    res[2] = (0.5*Q_minus[2]*t15*t6 + 0.5*Q_plus[2]*t12*t17 + 0.5*t18*t21*(p[0] + t20*(Q_minus[2]*Q_minus[2])) + 0.5*t21*t22*(p[0] + t23*(Q_plus[2]*Q_plus[2])));
    res[3] = (0.5*Q_minus[3]*t15*t5 + 0.5*Q_plus[3]*t11*t17 + 0.5*t18*t24*(p[0] + t20*(Q_minus[3]*Q_minus[3])) + 0.5*t22*t24*(p[0] + t23*(Q_plus[3]*Q_plus[3])));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 8> numerical_fluctuations(
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
    T t6 = (t2/(std::max((T)1e-14, Q_minus[1])));
    T t7 = t6*(Q_minus[2]*n[0] + Q_minus[3]*n[1]);
    T t8 = std::sqrt(p[0]);
    T t9 = t5*t8*(t2*t2*std::sqrt(t2));
    T t10 = (1.0/(std::max((T)1e-14, t3)));
    T t11 = (t4/(std::max((T)1e-14, Q_plus[1])));
    T t12 = t11*(Q_plus[2]*n[0] + Q_plus[3]*n[1]);
    T t13 = t10*t8*(t4*t4*std::sqrt(t4));
    T t14 = std::max(t10*std::fabs((t12 + t13)), std::max(t5*std::fabs((t7 + t9)), std::max(t10*std::fabs((t12 - t13)), t5*std::fabs((t7 - t9)))));
    T t15 = 0.5*t14*(t2 - t4);
    T t16 = p[0]*((Q_plus[1]*Q_plus[1]) - (t4*t4));
    T t17 = t14*(Q_minus[2]*t6 - Q_plus[2]*t11);
    T t18 = t14*(Q_minus[3]*t6 - Q_plus[3]*t11);
    T t19 = p[0]*((Q_minus[1]*Q_minus[1]) - (t2*t2));
    SimpleArray<T, 8> res;
    res[0] = 0.0;
    res[1] = (-t15);
    res[2] = ((-0.5*t17) - 0.5*n[0]*t16);
    res[3] = ((-0.5*t18) - 0.5*n[1]*t16);
    res[4] = 0.0;
    res[5] = t15;
    res[6] = (0.5*t17 + 0.5*n[0]*t19);
    res[7] = (0.5*t18 + 0.5*n[1]*t19);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 1> local_max_abs_eigenvalue(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = (1.0/(std::max((T)1e-14, Q[1])));
    T t1 = t0*std::sqrt(p[0])*std::sqrt(std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1])));
    T t2 = (Q[2]*n[0] + Q[3]*n[1]);
    SimpleArray<T, 1> res;
    res[0] = std::max(t0*std::fabs((t1 + t2)), t0*std::fabs((t1 - t2)));
    return res;
    }

};
