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
    T t2 = (1.0/(t1));
    T t3 = (-std::max(Q_minus[0], Q_plus[0]));
    T t4 = (Q_minus[0] + Q_minus[1] + t3);
    T t5 = std::max((T)0.0, t4);
    T t6 = t2*t5;
    T t7 = Q_minus[4]*n[1];
    T t8 = Q_plus[2]*n[0];
    T t9 = std::max((T)1e-14, Q_plus[1]);
    T t10 = (1.0/(t9));
    T t11 = (Q_plus[0] + Q_plus[1] + t3);
    T t12 = std::max((T)0.0, t11);
    T t13 = t10*t12;
    T t14 = Q_plus[4]*n[1];
    T t15 = std::sqrt(2.0);
    T t16 = 2.0*t15;
    T t17 = n[1]*t16;
    T t18 = (t5*t5*t5);
    T t19 = (1.0/(t1*t1));
    T t20 = (t19/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)))));
    T t21 = t18*t20;
    T t22 = t21*(Q_minus[3]*Q_minus[5] + 3.0*Q_minus[2]*Q_minus[4]);
    T t23 = (t12*t12*t12);
    T t24 = (1.0/(t9*t9));
    T t25 = (t24/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)))));
    T t26 = t23*t25;
    T t27 = t26*(Q_plus[3]*Q_plus[5] + 3.0*Q_plus[2]*Q_plus[4]);
    T t28 = (t5*t5);
    T t29 = 3.0*p[0];
    T t30 = t20*t5;
    T t31 = 6.0*t15;
    T t32 = t30*t31;
    T t33 = t16*t30;
    T t34 = (t12*t12);
    T t35 = t12*t25;
    T t36 = t31*t35;
    T t37 = t16*t35;
    T t38 = Q_minus[3]*n[0];
    T t39 = Q_plus[3]*n[0];
    T t40 = 0.5*n[1];
    T t41 = t21*(Q_minus[2]*Q_minus[5] + Q_minus[3]*Q_minus[4]);
    T t42 = t26*(Q_plus[2]*Q_plus[5] + Q_plus[3]*Q_plus[4]);
    T t43 = n[0]*t16;
    T t44 = Q_minus[5]*n[1];
    T t45 = Q_plus[5]*n[1];
    T t46 = 0.5*n[0];
    T t47 = t2*(t0 + t7);
    T t48 = std::max((T)1e-14, t4);
    T t49 = std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))));
    T t50 = (t5/(t48));
    T t51 = t10*(t14 + t8);
    T t52 = std::max((T)1e-14, t11);
    T t53 = std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))));
    T t54 = (t12/(t52));
    T t55 = std::max(t50*std::fabs((t47 + t49)), std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))));
    T t56 = 0.5*t55*(t5 - t12);
    T t57 = p[0]*((Q_plus[1]*Q_plus[1]) - t34);
    T t58 = Q_minus[2]*t6;
    T t59 = Q_plus[2]*t13;
    T t60 = t55*(t58 - t59);
    T t61 = (Q_minus[3]*t6 - Q_plus[3]*t13);
    T t62 = 4.0*t55;
    T t63 = t61*t62;
    T t64 = (t12 + t5);
    T t65 = (t15*t64/std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64))));
    T t66 = t65*(t58 + t59);
    T t67 = n[0]*t61;
    T t68 = (Q_minus[5]*t6 - Q_plus[5]*t13);
    T t69 = n[1]*t68;
    T t70 = (t66*t67 + t66*t69);
    T t71 = Q_minus[4]*t6;
    T t72 = Q_plus[4]*t13;
    T t73 = t55*(t71 - t72);
    T t74 = t62*t68;
    T t75 = t65*(t71 + t72);
    T t76 = (t67*t75 + t69*t75);
    T t77 = p[0]*((Q_minus[1]*Q_minus[1]) - t28);
    T a_t77 = (0.5*n[0]*w[14] + 0.5*n[1]*w[16]);
    T a_t76 = (0.125*w[11] + 0.125*w[17]);
    T a_t75 = (a_t76*t67 + a_t76*t69);
    T a_t74 = ((-0.125*w[11]) + 0.125*w[17]);
    T a_t73 = (0.5*w[16] - 0.5*w[10]);
    T a_t72 = (a_t75*t65 - a_t73*t55);
    T a_t71 = (a_t73*t55 + a_t75*t65);
    T a_t70 = (0.125*w[15] + 0.125*w[9]);
    T a_t69 = (a_t70*t66 + a_t76*t75);
    T a_t68 = (a_t69*n[1] + a_t74*t62);
    T a_t67 = (a_t70*t66 + a_t76*t75);
    T a_t66 = (a_t70*t67 + a_t70*t69);
    T a_t65 = (a_t66*(t58 + t59) + a_t75*(t71 + t72));
    T a_t64 = (0.5*(((T)1e-12 < 0.5*t64) ? (-(4.0*a_t65*t15*t64*(std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64))*(((T)0.0 < std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))) ? (0.5/std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))) : (T)0.0)/(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64))))) : (T)0.0) + (a_t65*t15/std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))) - (0.25*a_t65*t15*(t64*t64*t64*t64)*(((T)0.0 < std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))) ? (0.5/std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))) : (T)0.0)/(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))));
    T a_t63 = ((-0.125*w[9]) + 0.125*w[15]);
    T a_t62 = (a_t63*t61 + a_t74*t68);
    T a_t61 = (a_t63*t62 + a_t67*n[0]);
    T a_t60 = (0.5*w[14] - 0.5*w[8]);
    T a_t59 = (a_t66*t65 - a_t60*t55);
    T a_t58 = (a_t60*t55 + a_t66*t65);
    T a_t57 = ((-0.5*n[0]*w[8]) - 0.5*n[1]*w[10]);
    T a_t56 = (w[13] - w[7]);
    T a_t55 = (4.0*a_t62 + a_t56*(0.5*t5 - 0.5*t12) + a_t60*(t58 - t59) + a_t73*(t71 - t72));
    T a_t54 = (std::fabs((t51 + t53))*((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? (T)0.0 : ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0)) + std::fabs((t51 - t53))*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0) : (T)0.0));
    T a_t53 = ((-(((t51 - t53) < (T)0.0) ? (-t54*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0) : (T)0.0)) : t54*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0) : (T)0.0))) + (((t51 + t53) < (T)0.0) ? (-t54*((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? (T)0.0 : ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0))) : t54*((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? (T)0.0 : ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0))));
    T a_t52 = ((-(a_t54*t12/(t52*t52))) - (2.0*a_t53*p[0]*t23*(((T)0.0 < std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) ? (0.5/std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) : (T)0.0)/(t52*t52*t52)));
    T a_t51 = ((((t51 + t53) < (T)0.0) ? (-t54*((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? (T)0.0 : ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0))) : t54*((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? (T)0.0 : ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0))) + (((t51 - t53) < (T)0.0) ? (-t54*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0) : (T)0.0)) : t54*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0) : (T)0.0)));
    T a_t50 = (std::fabs((t47 + t49))*((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? (T)0.0 : a_t55) + std::fabs((t47 - t49))*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? (T)0.0 : ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0)));
    T a_t49 = ((-(((t47 - t49) < (T)0.0) ? (-t50*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? (T)0.0 : ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0))) : t50*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? (T)0.0 : ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0)))) + (((t47 + t49) < (T)0.0) ? (-t50*((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? (T)0.0 : a_t55)) : t50*((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? (T)0.0 : a_t55)));
    T a_t48 = ((-(a_t50*t5/(t48*t48))) - (2.0*a_t49*p[0]*t18*(((T)0.0 < std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) ? (0.5/std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) : (T)0.0)/(t48*t48*t48)));
    T a_t47 = ((((t47 + t49) < (T)0.0) ? (-t50*((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? (T)0.0 : a_t55)) : t50*((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? (T)0.0 : a_t55)) + (((t47 - t49) < (T)0.0) ? (-t50*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? (T)0.0 : ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0))) : t50*((t50*std::fabs((t47 - t49)) < t54*std::fabs((t51 - t53))) ? (T)0.0 : ((t54*std::fabs((t51 + t53)) < std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53)))) ? ((t50*std::fabs((t47 + t49)) < std::max(t54*std::fabs((t51 + t53)), std::max(t50*std::fabs((t47 - t49)), t54*std::fabs((t51 - t53))))) ? a_t55 : (T)0.0) : (T)0.0))));
    T a_t46 = (t15*t41*w[5] + t15*t42*w[5]);
    T a_t45 = (Q_plus[4]*t15*t26*w[5] + 2.0*a_t53*t24*(t39 + t45)*(((T)0.0 < std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) ? (0.5/std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) : (T)0.0));
    T a_t44 = (Q_minus[4]*t15*t21*w[5] + 2.0*a_t49*t19*(t38 + t44)*(((T)0.0 < std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) ? (0.5/std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) : (T)0.0));
    T a_t43 = (0.08333333333333333*t22*w[4] + 0.08333333333333333*t27*w[4]);
    T a_t42 = (t15*t40*w[3] + t15*t46*w[5]);
    T a_t41 = (t15*t40*w[3] + t15*t46*w[5]);
    T a_t40 = (t15*t41*w[3] + t15*t42*w[3]);
    T a_t39 = (Q_plus[2]*t15*t26*w[3] + 2.0*a_t53*t24*(t39 + t45)*(((T)0.0 < std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) ? (0.5/std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) : (T)0.0));
    T a_t38 = (Q_minus[2]*t15*t21*w[3] + 2.0*a_t49*t19*(t38 + t44)*(((T)0.0 < std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) ? (0.5/std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) : (T)0.0));
    T a_t37 = (0.08333333333333333*n[0]*t34*w[2]*(Q_plus[3]*Q_plus[3]) + 0.08333333333333333*n[1]*t34*w[4]*(Q_plus[5]*Q_plus[5]));
    T a_t36 = (0.08333333333333333*n[0]*t34*w[2]*(Q_plus[2]*Q_plus[2]) + 0.08333333333333333*n[1]*t34*w[4]*(Q_plus[4]*Q_plus[4]));
    T a_t35 = (a_t36*t31 + a_t37*t16);
    T a_t34 = ((-a_t57*p[0]) + 0.08333333333333333*n[0]*w[2]*(t29 + t36*(Q_plus[2]*Q_plus[2]) + t37*(Q_plus[3]*Q_plus[3])) + 0.08333333333333333*n[1]*w[4]*(t29 + t36*(Q_plus[4]*Q_plus[4]) + t37*(Q_plus[5]*Q_plus[5])));
    T a_t33 = (0.08333333333333333*n[0]*t28*w[2]*(Q_minus[3]*Q_minus[3]) + 0.08333333333333333*n[1]*t28*w[4]*(Q_minus[5]*Q_minus[5]));
    T a_t32 = (0.08333333333333333*n[0]*t28*w[2]*(Q_minus[2]*Q_minus[2]) + 0.08333333333333333*n[1]*t28*w[4]*(Q_minus[4]*Q_minus[4]));
    T a_t31 = (a_t32*t30 + a_t36*t35);
    T a_t30 = (a_t32*t31 + a_t33*t16);
    T a_t29 = (0.08333333333333333*n[0]*t28*w[2] + 0.08333333333333333*n[0]*t34*w[2] + 0.08333333333333333*n[1]*t28*w[4] + 0.08333333333333333*n[1]*t34*w[4]);
    T a_t28 = ((-a_t77*p[0]) + 0.08333333333333333*n[0]*w[2]*(t29 + t32*(Q_minus[2]*Q_minus[2]) + t33*(Q_minus[3]*Q_minus[3])) + 0.08333333333333333*n[1]*w[4]*(t29 + t32*(Q_minus[4]*Q_minus[4]) + t33*(Q_minus[5]*Q_minus[5])));
    T a_t27 = (0.08333333333333333*t17*w[2] + 0.08333333333333333*t43*w[4]);
    T a_t26 = (a_t27*(Q_plus[3]*Q_plus[5] + 3.0*Q_plus[2]*Q_plus[4]) + a_t42*(Q_plus[2]*Q_plus[5] + Q_plus[3]*Q_plus[4]) + Q_plus[2]*t15*t39*w[3] + Q_plus[4]*t15*t45*w[5]);
    T a_t25 = (a_t26*t23 + a_t35*t12);
    T a_t24 = ((a_t25/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) + a_t53*((t39 + t45)*(t39 + t45))*(((T)0.0 < std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) ? (0.5/std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) : (T)0.0));
    T a_t23 = (a_t26*t25 + (a_t53*p[0]*(((T)0.0 < std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) ? (0.5/std::sqrt((t24*((t39 + t45)*(t39 + t45)) + (p[0]*t23/(t52*t52))))) : (T)0.0)/(t52*t52)));
    T a_t22 = (0.08333333333333333*t17*w[2] + 0.08333333333333333*t43*w[4]);
    T a_t21 = (a_t22*(Q_minus[3]*Q_minus[5] + 3.0*Q_minus[2]*Q_minus[4]) + a_t41*(Q_minus[2]*Q_minus[5] + Q_minus[3]*Q_minus[4]) + Q_minus[2]*t15*t38*w[3] + Q_minus[4]*t15*t44*w[5]);
    T a_t20 = (a_t21*t18 + a_t30*t5);
    T a_t19 = ((a_t20/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) + a_t49*((t38 + t44)*(t38 + t44))*(((T)0.0 < std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) ? (0.5/std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) : (T)0.0));
    T a_t18 = (a_t21*t20 + (a_t49*p[0]*(((T)0.0 < std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) ? (0.5/std::sqrt((t19*((t38 + t44)*(t38 + t44)) + (p[0]*t18/(t48*t48))))) : (T)0.0)/(t48*t48)));
    T a_t17 = (0.08333333333333333*t22*w[2] + 0.08333333333333333*t27*w[2]);
    T a_t16 = (a_t17*n[1] + a_t33*t30 + a_t37*t35 + a_t43*n[0]);
    T a_t15 = (2.0*a_t16 + 6.0*a_t31 + w[3]*(t40*t41 + t40*t42 + Q_minus[2]*t21*t38 + Q_plus[2]*t26*t39) + w[5]*(t41*t46 + t42*t46 + Q_minus[4]*t21*t44 + Q_plus[4]*t26*t45) + (a_t65*t64/std::sqrt(((std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)*std::max((T)1e-12, 0.5*t64)) + 0.0625*(t64*t64*t64*t64)))));
    T a_t14 = (a_t51*t10 + 0.5*t13*w[1]);
    T a_t13 = (Q_plus[2]*a_t59 + Q_plus[4]*a_t72 + 0.5*t14*w[1] + 0.5*t8*w[1] - Q_plus[3]*a_t61 - Q_plus[5]*a_t68);
    T a_t12 = (a_t64 + a_t13*t10 + a_t35*t25 + (a_t54/(t52)) + 2.0*a_t34*t12 + 3.0*a_t23*(t12*t12) - 0.5*a_t56*t55 - (4.0*a_t25*t24*(t12*t12*t12)*(((T)0.0 < std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) ? (0.5/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) : (T)0.0)/(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))));
    T a_t11 = ((((T)0.0 < t11) ? a_t12 : (T)0.0) + (((T)1e-12 < t11) ? (-(4.0*a_t25*t24*(std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))*(((T)0.0 < std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) ? (0.5/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) : (T)0.0)/(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)))))) : (T)0.0) + (((T)1e-14 < t11) ? a_t52 : (T)0.0));
    T a_t10 = (a_t13*t12 + a_t51*(t14 + t8));
    T a_t9 = ((-(a_t10/(t9*t9))) - (2.0*a_t24/(t9*t9*t9)));
    T a_t8 = (a_t51*t10 + 0.5*t13*w[1]);
    T a_t7 = (a_t47*t2 + 0.5*t6*w[1]);
    T a_t6 = (Q_minus[2]*a_t58 + Q_minus[3]*a_t61 + Q_minus[4]*a_t71 + Q_minus[5]*a_t68 + 0.5*t0*w[1] + 0.5*t7*w[1]);
    T a_t5 = (a_t64 + a_t30*t20 + (a_t50/(t48)) + a_t6*t2 + 0.5*a_t56*t55 + 2.0*a_t28*t5 + 3.0*a_t18*(t5*t5) - (4.0*a_t20*t19*(t5*t5*t5)*(((T)0.0 < std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) ? (0.5/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) : (T)0.0)/(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))));
    T a_t4 = ((((T)0.0 < t4) ? a_t5 : (T)0.0) + (((T)1e-12 < t4) ? (-(4.0*a_t20*t19*(std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))*(((T)0.0 < std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) ? (0.5/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) : (T)0.0)/(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)))))) : (T)0.0) + (((T)1e-14 < t4) ? a_t48 : (T)0.0));
    T a_t3 = (a_t11 + a_t4);
    T a_t2 = (a_t47*(t0 + t7) + a_t6*t5);
    T a_t1 = ((-(a_t2/(t1*t1))) - (2.0*a_t19/(t1*t1*t1)));
    T a_t0 = (a_t47*t2 + 0.5*t6*w[1]);
    g[0] = (a_t4 + ((Q_minus[0] < Q_plus[0]) ? (T)0.0 : (-a_t3)));
    g[1] = (a_t4 + 2.0*Q_minus[1]*a_t77*p[0] + (((T)1e-14 < Q_minus[1]) ? a_t1 : (T)0.0));
    g[2] = (a_t0*n[0] + a_t58*t6 + Q_minus[5]*a_t41*t21 + 3.0*Q_minus[4]*a_t22*t21 + t15*t21*t38*w[3] + 0.16666666666666666*Q_minus[2]*n[0]*t28*t32*w[2]);
    g[3] = (a_t38*n[0] + a_t61*t6 + Q_minus[4]*a_t41*t21 + Q_minus[5]*a_t22*t21 + 0.16666666666666666*Q_minus[3]*n[0]*t28*t33*w[2]);
    g[4] = (a_t7*n[1] + a_t71*t6 + Q_minus[3]*a_t41*t21 + 3.0*Q_minus[2]*a_t22*t21 + t15*t21*t44*w[5] + 0.16666666666666666*Q_minus[4]*n[1]*t28*t32*w[4]);
    g[5] = (a_t44*n[1] + a_t68*t6 + Q_minus[2]*a_t41*t21 + Q_minus[3]*a_t22*t21 + 0.16666666666666666*Q_minus[5]*n[1]*t28*t33*w[4]);
    g[6] = (a_t11 + ((Q_minus[0] < Q_plus[0]) ? (-a_t3) : (T)0.0));
    g[7] = (a_t11 + 2.0*Q_plus[1]*a_t57*p[0] + (((T)1e-14 < Q_plus[1]) ? a_t9 : (T)0.0));
    g[8] = (a_t59*t13 + a_t8*n[0] + Q_plus[5]*a_t42*t26 + 3.0*Q_plus[4]*a_t27*t26 + t15*t26*t39*w[3] + 0.16666666666666666*Q_plus[2]*n[0]*t34*t36*w[2]);
    g[9] = (a_t39*n[0] - a_t61*t13 + Q_plus[4]*a_t42*t26 + Q_plus[5]*a_t27*t26 + 0.16666666666666666*Q_plus[3]*n[0]*t34*t37*w[2]);
    g[10] = (a_t14*n[1] + a_t72*t13 + Q_plus[3]*a_t42*t26 + 3.0*Q_plus[2]*a_t27*t26 + t15*t26*t45*w[5] + 0.16666666666666666*Q_plus[4]*n[1]*t34*t36*w[4]);
    g[11] = (a_t45*n[1] - a_t68*t13 + Q_plus[2]*a_t42*t26 + Q_plus[3]*a_t27*t26 + 0.16666666666666666*Q_plus[5]*n[1]*t34*t37*w[4]);
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
