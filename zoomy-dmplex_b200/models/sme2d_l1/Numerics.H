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
#include "Model.H"

template <typename T>
struct Numerics {
    static constexpr int n_dof_q = 6;
    PORTABLE_FN static inline SimpleArray<T, 6> numerical_flux(
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
    T t6 = Q_minus[4]*n[1];
    T t7 = std::max((T)1e-14, Q_plus[1]);
    T t8 = (Q_plus[0] + Q_plus[1] + t1);
    T t9 = std::max((T)0.0, t8);
    T t10 = (t9/(t7));
    T t11 = Q_plus[2]*n[0];
    T t12 = Q_plus[4]*n[1];
    T t13 = std::sqrt(2.0);
    T t14 = 2.0*t13;
    T t15 = n[1]*t14;
    T t16 = (1.0/((t0*t0)*std::sqrt(((t3*t3*t3*t3) + (std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2))))));
    T t17 = t16*(t3*t3*t3);
    T t18 = t17*(Q_minus[3]*Q_minus[5] + 3.0*Q_minus[2]*Q_minus[4]);
    T t19 = (1.0/((t7*t7)*std::sqrt(((t9*t9*t9*t9) + (std::max((T)1e-12, t8)*std::max((T)1e-12, t8)*std::max((T)1e-12, t8)*std::max((T)1e-12, t8))))));
    T t20 = t19*(t9*t9*t9);
    T t21 = t20*(Q_plus[3]*Q_plus[5] + 3.0*Q_plus[2]*Q_plus[4]);
    T t22 = (t3*t3);
    T t23 = 3.0*p[0];
    T t24 = t16*t3;
    T t25 = 6.0*t13;
    T t26 = t24*t25;
    T t27 = t14*t24;
    T t28 = (t9*t9);
    T t29 = t19*t9;
    T t30 = t25*t29;
    T t31 = t14*t29;
    T t32 = 0.5*n[1];
    T t33 = t17*(Q_minus[2]*Q_minus[5] + Q_minus[3]*Q_minus[4]);
    T t34 = t20*(Q_plus[2]*Q_plus[5] + Q_plus[3]*Q_plus[4]);
    T t35 = n[0]*t14;
    T t36 = 0.5*n[0];
    SimpleArray<T, 6> res;
    res[0] = 0.0;
    res[1] = (0.5*t10*t11 + 0.5*t10*t12 + 0.5*t4*t5 + 0.5*t4*t6);
    res[2] = (0.08333333333333333*t15*t18 + 0.08333333333333333*t15*t21 + 0.08333333333333333*n[0]*t22*(t23 + t26*(Q_minus[2]*Q_minus[2]) + t27*(Q_minus[3]*Q_minus[3])) + 0.08333333333333333*n[0]*t28*(t23 + t30*(Q_plus[2]*Q_plus[2]) + t31*(Q_plus[3]*Q_plus[3])));
    res[3] = t13*(t32*t33 + t32*t34 + Q_minus[3]*t17*t5 + Q_plus[3]*t11*t20);
    res[4] = (0.08333333333333333*t18*t35 + 0.08333333333333333*t21*t35 + 0.08333333333333333*n[1]*t22*(t23 + t26*(Q_minus[4]*Q_minus[4]) + t27*(Q_minus[5]*Q_minus[5])) + 0.08333333333333333*n[1]*t28*(t23 + t30*(Q_plus[4]*Q_plus[4]) + t31*(Q_plus[5]*Q_plus[5])));
    res[5] = t13*(t33*t36 + t34*t36 + Q_minus[5]*t17*t6 + Q_plus[5]*t12*t20);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> numerical_fluctuations(
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
    T t5 = std::max((T)1e-14, Q_minus[1]);
    T t6 = (1.0/(t5));
    T t7 = t6*(Q_minus[2]*n[0] + Q_minus[4]*n[1]);
    T t8 = std::max((T)1e-14, t1);
    T t9 = std::sqrt(((((Q_minus[3]*n[0] + Q_minus[5]*n[1])*(Q_minus[3]*n[0] + Q_minus[5]*n[1]))/(t5*t5)) + (p[0]*(t2*t2*t2)/(t8*t8))));
    T t10 = (t2/(t8));
    T t11 = std::max((T)1e-14, Q_plus[1]);
    T t12 = (1.0/(t11));
    T t13 = t12*(Q_plus[2]*n[0] + Q_plus[4]*n[1]);
    T t14 = std::max((T)1e-14, t3);
    T t15 = std::sqrt(((((Q_plus[3]*n[0] + Q_plus[5]*n[1])*(Q_plus[3]*n[0] + Q_plus[5]*n[1]))/(t11*t11)) + (p[0]*(t4*t4*t4)/(t14*t14))));
    T t16 = (t4/(t14));
    T t17 = std::max(t10*std::fabs((t7 + t9)), std::max(t16*std::fabs((t13 + t15)), std::max(t10*std::fabs((t7 - t9)), t16*std::fabs((t13 - t15)))));
    T t18 = 0.5*t17*(t2 - t4);
    T t19 = p[0]*((Q_plus[1]*Q_plus[1]) - (t4*t4));
    T t20 = t2*t6;
    T t21 = Q_minus[2]*t20;
    T t22 = t12*t4;
    T t23 = Q_plus[2]*t22;
    T t24 = t17*(t21 - t23);
    T t25 = (Q_minus[3]*t20 - Q_plus[3]*t22);
    T t26 = 4.0*t17;
    T t27 = t25*t26;
    T t28 = (t2 + t4);
    T t29 = (t28*std::sqrt(2.0)/std::sqrt(((std::max((T)1e-12, 0.5*t28)*std::max((T)1e-12, 0.5*t28)*std::max((T)1e-12, 0.5*t28)*std::max((T)1e-12, 0.5*t28)) + 0.0625*(t28*t28*t28*t28))));
    T t30 = t29*(t21 + t23);
    T t31 = n[0]*t25;
    T t32 = (Q_minus[5]*t20 - Q_plus[5]*t22);
    T t33 = n[1]*t32;
    T t34 = (t30*t31 + t30*t33);
    T t35 = Q_minus[4]*t20;
    T t36 = Q_plus[4]*t22;
    T t37 = t17*(t35 - t36);
    T t38 = t26*t32;
    T t39 = t29*(t35 + t36);
    T t40 = (t31*t39 + t33*t39);
    T t41 = p[0]*((Q_minus[1]*Q_minus[1]) - (t2*t2));
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = (-t18);
    res[2] = ((-0.5*t24) - 0.5*n[0]*t19);
    res[3] = ((-0.125*t27) + 0.125*t34);
    res[4] = ((-0.5*t37) - 0.5*n[1]*t19);
    res[5] = ((-0.125*t38) + 0.125*t40);
    res[6] = 0.0;
    res[7] = t18;
    res[8] = (0.5*t24 + 0.5*n[0]*t41);
    res[9] = (0.125*t27 + 0.125*t34);
    res[10] = (0.5*t37 + 0.5*n[1]*t41);
    res[11] = (0.125*t38 + 0.125*t40);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 1> local_max_abs_eigenvalue(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = std::max((T)1e-14, Q[1]);
    T t1 = (1.0/(t0));
    T t2 = std::sqrt((((Q[3]*n[0] + Q[5]*n[1])*(Q[3]*n[0] + Q[5]*n[1])) + (p[0]*std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1]))/(t0*t0))));
    T t3 = (Q[2]*n[0] + Q[4]*n[1]);
    SimpleArray<T, 1> res;
    res[0] = std::max(t1*std::fabs((t2 + t3)), t1*std::fabs((t2 - t3)));
    return res;
    }

};
