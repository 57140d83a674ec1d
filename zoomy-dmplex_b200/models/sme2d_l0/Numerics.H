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

    PORTABLE_FN static inline void numerical_flux_fluct_vjp(
        const T* Q_minus,
        const T* Q_plus,
        const T* Qaux_minus,
        const T* Qaux_plus,
        const T* p,
        const T* n,
        const T* w,
        T* g)
    {
    T t0 = Q_minus[2]*n[0];
    T t1 = std::max((T)1e-14, Q_minus[1]);
    T t2 = (-std::max(Q_minus[0], Q_plus[0]));
    T t3 = (Q_minus[0] + Q_minus[1] + t2);
    T t4 = std::max((T)0.0, t3);
    T t5 = (t4/(t1));
    T t6 = Q_minus[3]*n[1];
    T t7 = Q_plus[2]*n[0];
    T t8 = std::max((T)1e-14, Q_plus[1]);
    T t9 = (Q_plus[0] + Q_plus[1] + t2);
    T t10 = std::max((T)0.0, t9);
    T t11 = (t10/(t8));
    T t12 = Q_plus[3]*n[1];
    T t13 = std::sqrt(2.0);
    T t14 = (1.0/((t1*t1)*std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))));
    T t15 = t13*t14*(t4*t4*t4);
    T t16 = (1.0/((t8*t8)*std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))));
    T t17 = t13*t16*(t10*t10*t10);
    T t18 = (t4*t4);
    T t19 = 2.0*t13;
    T t20 = t14*t19*t4;
    T t21 = 0.5*n[0];
    T t22 = (t10*t10);
    T t23 = t10*t16*t19;
    T t24 = 0.5*n[1];
    T t25 = (1.0/(std::max((T)1e-14, t3)));
    T t26 = t5*(t0 + t6);
    T t27 = std::sqrt(p[0]);
    T t28 = t25*t27*(t4*t4*std::sqrt(t4));
    T t29 = (1.0/(std::max((T)1e-14, t9)));
    T t30 = t11*(t12 + t7);
    T t31 = t27*t29*(t10*t10*std::sqrt(t10));
    T t32 = std::max(t25*std::fabs((t26 + t28)), std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))));
    T t33 = 0.5*t32*(t4 - t10);
    T t34 = p[0]*((Q_plus[1]*Q_plus[1]) - t22);
    T t35 = t32*(Q_minus[2]*t5 - Q_plus[2]*t11);
    T t36 = t32*(Q_minus[3]*t5 - Q_plus[3]*t11);
    T t37 = p[0]*((Q_minus[1]*Q_minus[1]) - t18);
    T a_t37 = (0.5*n[0]*w[10] + 0.5*n[1]*w[11]);
    T a_t36 = (0.5*w[11] - 0.5*w[7]);
    T a_t35 = (0.5*w[10] - 0.5*w[6]);
    T a_t34 = ((-0.5*n[0]*w[6]) - 0.5*n[1]*w[7]);
    T a_t33 = (w[9] - w[5]);
    T a_t32 = (a_t33*(0.5*t4 - 0.5*t10) + a_t35*(Q_minus[2]*t5 - Q_plus[2]*t11) + a_t36*(Q_minus[3]*t5 - Q_plus[3]*t11));
    T a_t31 = ((-(((t30 - t31) < (T)0.0) ? (-t29*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0) : (T)0.0)) : t29*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0) : (T)0.0))) + (((t30 + t31) < (T)0.0) ? (-t29*((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? (T)0.0 : ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0))) : t29*((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? (T)0.0 : ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0))));
    T a_t30 = ((((t30 + t31) < (T)0.0) ? (-t29*((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? (T)0.0 : ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0))) : t29*((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? (T)0.0 : ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0))) + (((t30 - t31) < (T)0.0) ? (-t29*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0) : (T)0.0)) : t29*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0) : (T)0.0)));
    T a_t29 = (std::fabs((t30 + t31))*((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? (T)0.0 : ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0)) + std::fabs((t30 - t31))*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0) : (T)0.0) + a_t31*t27*(t10*t10*std::sqrt(t10)));
    T a_t28 = ((-(((t26 - t28) < (T)0.0) ? (-t25*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? (T)0.0 : ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0))) : t25*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? (T)0.0 : ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0)))) + (((t26 + t28) < (T)0.0) ? (-t25*((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? (T)0.0 : a_t32)) : t25*((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? (T)0.0 : a_t32)));
    T a_t27 = (a_t28*t25*(t4*t4*std::sqrt(t4)) + a_t31*t29*(t10*t10*std::sqrt(t10)));
    T a_t26 = ((((t26 + t28) < (T)0.0) ? (-t25*((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? (T)0.0 : a_t32)) : t25*((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? (T)0.0 : a_t32)) + (((t26 - t28) < (T)0.0) ? (-t25*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? (T)0.0 : ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0))) : t25*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? (T)0.0 : ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0))));
    T a_t25 = (std::fabs((t26 + t28))*((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? (T)0.0 : a_t32) + std::fabs((t26 - t28))*((t25*std::fabs((t26 - t28)) < t29*std::fabs((t30 - t31))) ? (T)0.0 : ((t29*std::fabs((t30 + t31)) < std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31)))) ? ((t25*std::fabs((t26 + t28)) < std::max(t29*std::fabs((t30 + t31)), std::max(t25*std::fabs((t26 - t28)), t29*std::fabs((t30 - t31))))) ? a_t32 : (T)0.0) : (T)0.0)) + a_t28*t27*(t4*t4*std::sqrt(t4)));
    T a_t24 = (0.5*t18*w[3]*(p[0] + t20*(Q_minus[3]*Q_minus[3])) + 0.5*t22*w[3]*(p[0] + t23*(Q_plus[3]*Q_plus[3])));
    T a_t23 = (0.5*t21*t22*w[2]*(Q_plus[2]*Q_plus[2]) + 0.5*t22*t24*w[3]*(Q_plus[3]*Q_plus[3]));
    T a_t22 = ((-a_t34*p[0]) + 0.5*t21*w[2]*(p[0] + t23*(Q_plus[2]*Q_plus[2])) + 0.5*t24*w[3]*(p[0] + t23*(Q_plus[3]*Q_plus[3])));
    T a_t21 = (0.5*t18*w[2]*(p[0] + t20*(Q_minus[2]*Q_minus[2])) + 0.5*t22*w[2]*(p[0] + t23*(Q_plus[2]*Q_plus[2])));
    T a_t20 = (0.5*t18*t21*w[2]*(Q_minus[2]*Q_minus[2]) + 0.5*t18*t24*w[3]*(Q_minus[3]*Q_minus[3]));
    T a_t19 = (a_t20*t14*t4 + a_t23*t10*t16);
    T a_t18 = ((-a_t37*p[0]) + 0.5*t21*w[2]*(p[0] + t20*(Q_minus[2]*Q_minus[2])) + 0.5*t24*w[3]*(p[0] + t20*(Q_minus[3]*Q_minus[3])));
    T a_t17 = (0.5*Q_plus[2]*t12*w[2] + 0.5*Q_plus[3]*t7*w[3]);
    T a_t16 = (a_t17*t13*(t10*t10*t10) + a_t23*t10*t19);
    T a_t15 = (0.5*Q_minus[2]*t6*w[2] + 0.5*Q_minus[3]*t0*w[3]);
    T a_t14 = (a_t15*t13*(t4*t4*t4) + a_t20*t19*t4);
    T a_t13 = (2.0*a_t19 + a_t15*t14*(t4*t4*t4) + a_t17*t16*(t10*t10*t10));
    T a_t12 = (a_t30*t11 + 0.5*t11*w[1] + 0.5*Q_plus[2]*t17*w[2]);
    T a_t11 = (a_t30*(t12 + t7) + 0.5*t12*w[1] + 0.5*t7*w[1] - Q_plus[2]*a_t35*t32 - Q_plus[3]*a_t36*t32);
    T a_t10 = ((a_t11/(t8)) + 2.0*a_t22*t10 - 0.5*a_t33*t32 + a_t23*t16*t19 + a_t31*t27*t29*(2.0*(t10*std::sqrt(t10)) + (t10*t10)*(((T)0.0 < std::sqrt(t10)) ? (0.5/std::sqrt(t10)) : (T)0.0)) + 3.0*a_t17*t13*t16*(t10*t10) - (4.0*a_t16*(t10*t10*t10)*(((T)0.0 < std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))) ? (0.5/std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))) : (T)0.0)/((t8*t8)*(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)))))));
    T a_t9 = ((((T)0.0 < t9) ? a_t10 : (T)0.0) + (((T)1e-12 < t9) ? (-(4.0*a_t16*(std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))*(((T)0.0 < std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))) ? (0.5/std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))) : (T)0.0)/((t8*t8)*(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9))))))) : (T)0.0) + (((T)1e-14 < t9) ? (-(a_t29/(std::max((T)1e-14, t9)*std::max((T)1e-14, t9)))) : (T)0.0));
    T a_t8 = ((-(a_t11*t10/(t8*t8))) - (2.0*a_t16/((t8*t8*t8)*std::sqrt(((t10*t10*t10*t10) + (std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)*std::max((T)1e-12, t9)))))));
    T a_t7 = (a_t30*t11 + 0.5*t11*w[1] + 0.5*Q_plus[3]*t17*w[3]);
    T a_t6 = (a_t26*t5 + 0.5*t5*w[1] + 0.5*Q_minus[2]*t15*w[2]);
    T a_t5 = (a_t26*(t0 + t6) + 0.5*t0*w[1] + 0.5*t6*w[1] + Q_minus[2]*a_t35*t32 + Q_minus[3]*a_t36*t32);
    T a_t4 = ((a_t5/(t1)) + 0.5*a_t33*t32 + 2.0*a_t18*t4 + a_t20*t14*t19 + a_t28*t25*t27*(2.0*(t4*std::sqrt(t4)) + (t4*t4)*(((T)0.0 < std::sqrt(t4)) ? (0.5/std::sqrt(t4)) : (T)0.0)) + 3.0*a_t15*t13*t14*(t4*t4) - (4.0*a_t14*(t4*t4*t4)*(((T)0.0 < std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))) ? (0.5/std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))) : (T)0.0)/((t1*t1)*(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)))))));
    T a_t3 = ((((T)0.0 < t3) ? a_t4 : (T)0.0) + (((T)1e-12 < t3) ? (-(4.0*a_t14*(std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))*(((T)0.0 < std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))) ? (0.5/std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))) : (T)0.0)/((t1*t1)*(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3))))))) : (T)0.0) + (((T)1e-14 < t3) ? (-(a_t25/(std::max((T)1e-14, t3)*std::max((T)1e-14, t3)))) : (T)0.0));
    T a_t2 = (a_t3 + a_t9);
    T a_t1 = ((-(a_t5*t4/(t1*t1))) - (2.0*a_t14/((t1*t1*t1)*std::sqrt(((t4*t4*t4*t4) + (std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)*std::max((T)1e-12, t3)))))));
    T a_t0 = (a_t26*t5 + 0.5*t5*w[1] + 0.5*Q_minus[3]*t15*w[3]);
    g[0] = (a_t3 + ((Q_minus[0] < Q_plus[0]) ? (T)0.0 : (-a_t2)));
    g[1] = (a_t3 + 2.0*Q_minus[1]*a_t37*p[0] + (((T)1e-14 < Q_minus[1]) ? a_t1 : (T)0.0));
    g[2] = (a_t0*n[0] + a_t35*t32*t5 + 0.5*t15*t6*w[2] + Q_minus[2]*t18*t20*t21*w[2]);
    g[3] = (a_t6*n[1] + a_t36*t32*t5 + 0.5*t0*t15*w[3] + Q_minus[3]*t18*t20*t24*w[3]);
    g[4] = (a_t9 + ((Q_minus[0] < Q_plus[0]) ? (-a_t2) : (T)0.0));
    g[5] = (a_t9 + 2.0*Q_plus[1]*a_t34*p[0] + (((T)1e-14 < Q_plus[1]) ? a_t8 : (T)0.0));
    g[6] = (a_t7*n[0] + 0.5*t12*t17*w[2] - a_t35*t11*t32 + Q_plus[2]*t21*t22*t23*w[2]);
    g[7] = (a_t12*n[1] + 0.5*t17*t7*w[3] - a_t36*t11*t32 + Q_plus[3]*t22*t23*t24*w[3]);
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
