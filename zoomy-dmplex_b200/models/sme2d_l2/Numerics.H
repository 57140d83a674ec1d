#pragma once
// Generated by models/gen_sme.py (sme2d_l2: dim=2 level=2). Do not edit by hand.
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
    static constexpr int n_dof_q = 8;
    PORTABLE_FN static inline SimpleArray<T, 8> numerical_flux(
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
    T t5 = std::max((T)1e-14, Q_plus[1]);
    T t6 = (Q_plus[0] + Q_plus[1] + t1);
    T t7 = std::max((T)0.0, t6);
    T t8 = (t7/(t5));
    T t9 = (1.0/((t0*t0)*std::sqrt(((t3*t3*t3*t3) + (std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2)*std::max((T)1e-12, t2))))));
    T t10 = t9*(t3*t3*t3);
    T t11 = n[1]*t10;
    T t12 = 2.0*t11;
    T t13 = std::sqrt(2.0);
    T t14 = Q_minus[3]*Q_minus[6];
    T t15 = Q_minus[4]*Q_minus[7];
    T t16 = t13*(3.0*t15 + 5.0*t14 + 15.0*Q_minus[2]*Q_minus[5]);
    T t17 = (1.0/((t5*t5)*std::sqrt(((t7*t7*t7*t7) + (std::max((T)1e-12, t6)*std::max((T)1e-12, t6)*std::max((T)1e-12, t6)*std::max((T)1e-12, t6))))));
    T t18 = t17*(t7*t7*t7);
    T t19 = n[1]*t18;
    T t20 = 2.0*t19;
    T t21 = Q_plus[3]*Q_plus[6];
    T t22 = Q_plus[4]*Q_plus[7];
    T t23 = t13*(3.0*t22 + 5.0*t21 + 15.0*Q_plus[2]*Q_plus[5]);
    T t24 = (t3*t3);
    T t25 = 15.0*p[0];
    T t26 = t3*t9;
    T t27 = t13*t26;
    T t28 = 30.0*t27;
    T t29 = (Q_minus[3]*Q_minus[3]);
    T t30 = 10.0*t27;
    T t31 = (Q_minus[4]*Q_minus[4]);
    T t32 = 6.0*t13;
    T t33 = t26*t32;
    T t34 = (t7*t7);
    T t35 = t17*t7;
    T t36 = t13*t35;
    T t37 = 30.0*t36;
    T t38 = (Q_plus[3]*Q_plus[3]);
    T t39 = 10.0*t36;
    T t40 = (Q_plus[4]*Q_plus[4]);
    T t41 = t32*t35;
    T t42 = 5.0*Q_minus[2];
    T t43 = 2.0*Q_minus[4];
    T t44 = n[0]*t10;
    T t45 = 2.0*t44;
    T t46 = 5.0*Q_plus[2];
    T t47 = 2.0*Q_plus[4];
    T t48 = n[0]*t18;
    T t49 = 2.0*t48;
    T t50 = 5.0*Q_minus[5];
    T t51 = 2.0*Q_minus[7];
    T t52 = (Q_minus[3]*t50 + Q_minus[3]*t51 + Q_minus[6]*t42 + Q_minus[6]*t43);
    T t53 = 5.0*Q_plus[5];
    T t54 = 2.0*Q_plus[7];
    T t55 = (Q_plus[3]*t53 + Q_plus[3]*t54 + Q_plus[6]*t46 + Q_plus[6]*t47);
    T t56 = 0.1*t13;
    T t57 = 21.0*Q_minus[2];
    T t58 = 21.0*Q_plus[2];
    T t59 = 21.0*Q_minus[5];
    T t60 = (6.0*t15 + 14.0*t14 + Q_minus[4]*t59 + Q_minus[7]*t57);
    T t61 = 21.0*Q_plus[5];
    T t62 = (6.0*t22 + 14.0*t21 + Q_plus[4]*t61 + Q_plus[7]*t58);
    T t63 = 0.023809523809523808*t13;
    T t64 = (Q_minus[6]*Q_minus[6]);
    T t65 = (Q_minus[7]*Q_minus[7]);
    T t66 = (Q_plus[6]*Q_plus[6]);
    T t67 = (Q_plus[7]*Q_plus[7]);
    SimpleArray<T, 8> res;
    res[0] = 0.0;
    res[1] = (0.5*Q_minus[2]*n[0]*t4 + 0.5*Q_minus[5]*n[1]*t4 + 0.5*Q_plus[2]*n[0]*t8 + 0.5*Q_plus[5]*n[1]*t8);
    res[2] = (0.016666666666666666*t12*t16 + 0.016666666666666666*t20*t23 + 0.016666666666666666*n[0]*t24*(t25 + t28*(Q_minus[2]*Q_minus[2]) + t29*t30 + t31*t33) + 0.016666666666666666*n[0]*t34*(t25 + t37*(Q_plus[2]*Q_plus[2]) + t38*t39 + t40*t41));
    res[3] = t56*(t11*t52 + t19*t55 + Q_minus[3]*t45*(t42 + t43) + Q_plus[3]*t49*(t46 + t47));
    res[4] = t63*(t11*t60 + t19*t62 + t45*(3.0*t31 + 7.0*t29 + Q_minus[4]*t57) + t49*(3.0*t40 + 7.0*t38 + Q_plus[4]*t58));
    res[5] = (0.016666666666666666*t16*t45 + 0.016666666666666666*t23*t49 + 0.016666666666666666*n[1]*t24*(t25 + t28*(Q_minus[5]*Q_minus[5]) + t30*t64 + t33*t65) + 0.016666666666666666*n[1]*t34*(t25 + t37*(Q_plus[5]*Q_plus[5]) + t39*t66 + t41*t67));
    res[6] = t56*(t44*t52 + t48*t55 + Q_minus[6]*t12*(t50 + t51) + Q_plus[6]*t20*(t53 + t54));
    res[7] = t63*(t12*(3.0*t65 + 7.0*t64 + Q_minus[7]*t59) + t20*(3.0*t67 + 7.0*t66 + Q_plus[7]*t61) + t44*t60 + t48*t62);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 16> numerical_fluctuations(
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
    T t7 = t6*(Q_minus[2]*n[0] + Q_minus[5]*n[1]);
    T t8 = (1.0/(t5*t5));
    T t9 = std::max((T)1e-14, t1);
    T t10 = std::sqrt((t8*((Q_minus[3]*n[0] + Q_minus[6]*n[1])*(Q_minus[3]*n[0] + Q_minus[6]*n[1])) + 0.6*t8*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*(t2*t2*t2)/(t9*t9))));
    T t11 = (t2/(t9));
    T t12 = std::max((T)1e-14, Q_plus[1]);
    T t13 = (1.0/(t12));
    T t14 = t13*(Q_plus[2]*n[0] + Q_plus[5]*n[1]);
    T t15 = (1.0/(t12*t12));
    T t16 = std::max((T)1e-14, t3);
    T t17 = std::sqrt((t15*((Q_plus[3]*n[0] + Q_plus[6]*n[1])*(Q_plus[3]*n[0] + Q_plus[6]*n[1])) + 0.6*t15*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*(t4*t4*t4)/(t16*t16))));
    T t18 = (t4/(t16));
    T t19 = std::max(t11*std::fabs((t10 + t7)), std::max(t18*std::fabs((t14 + t17)), std::max(t11*std::fabs((t10 - t7)), t18*std::fabs((t14 - t17)))));
    T t20 = 0.5*t19*(t2 - t4);
    T t21 = p[0]*((Q_plus[1]*Q_plus[1]) - (t4*t4));
    T t22 = t2*t6;
    T t23 = Q_minus[2]*t22;
    T t24 = t13*t4;
    T t25 = Q_plus[2]*t24;
    T t26 = t19*(t23 - t25);
    T t27 = Q_minus[3]*t22;
    T t28 = Q_plus[3]*t24;
    T t29 = (t27 - t28);
    T t30 = 20.0*t19;
    T t31 = t29*t30;
    T t32 = (t27 + t28);
    T t33 = Q_minus[4]*t22;
    T t34 = Q_plus[4]*t24;
    T t35 = (-t34);
    T t36 = (t33 + t35);
    T t37 = (t2 + t4);
    T t38 = (t37*std::sqrt(2.0)/std::sqrt(((std::max((T)1e-12, 0.5*t37)*std::max((T)1e-12, 0.5*t37)*std::max((T)1e-12, 0.5*t37)*std::max((T)1e-12, 0.5*t37)) + 0.0625*(t37*t37*t37*t37))));
    T t39 = n[0]*t38;
    T t40 = t36*t39;
    T t41 = (t35 - t33 + 5.0*t23 + 5.0*t25);
    T t42 = t29*t39;
    T t43 = Q_minus[7]*t22;
    T t44 = Q_plus[7]*t24;
    T t45 = (-t44);
    T t46 = (t43 + t45);
    T t47 = n[1]*t38;
    T t48 = t46*t47;
    T t49 = Q_minus[6]*t22;
    T t50 = Q_plus[6]*t24;
    T t51 = (t49 - t50);
    T t52 = t47*t51;
    T t53 = (t32*t40 + t32*t48 + t41*t42 + t41*t52);
    T t54 = 28.0*t19;
    T t55 = t36*t54;
    T t56 = (t33 + t34 + 7.0*t23 + 7.0*t25);
    T t57 = 7.0*t32;
    T t58 = (t40*t56 + t42*t57 + t48*t56 + t52*t57);
    T t59 = Q_minus[5]*t22;
    T t60 = Q_plus[5]*t24;
    T t61 = t19*(t59 - t60);
    T t62 = t30*t51;
    T t63 = (t45 - t43 + 5.0*t59 + 5.0*t60);
    T t64 = (t49 + t50);
    T t65 = (t40*t64 + t42*t63 + t48*t64 + t52*t63);
    T t66 = t46*t54;
    T t67 = (t43 + t44 + 7.0*t59 + 7.0*t60);
    T t68 = 7.0*t64;
    T t69 = (t40*t67 + t42*t68 + t48*t67 + t52*t68);
    T t70 = p[0]*((Q_minus[1]*Q_minus[1]) - (t2*t2));
    SimpleArray<T, 16> res;
    res[0] = 0.0;
    res[1] = (-t20);
    res[2] = ((-0.5*t26) - 0.5*n[0]*t21);
    res[3] = ((-0.025*t31) + 0.025*t53);
    res[4] = ((-0.017857142857142856*t55) + 0.017857142857142856*t58);
    res[5] = ((-0.5*t61) - 0.5*n[1]*t21);
    res[6] = ((-0.025*t62) + 0.025*t65);
    res[7] = ((-0.017857142857142856*t66) + 0.017857142857142856*t69);
    res[8] = 0.0;
    res[9] = t20;
    res[10] = (0.5*t26 + 0.5*n[0]*t70);
    res[11] = (0.025*t31 + 0.025*t53);
    res[12] = (0.017857142857142856*t55 + 0.017857142857142856*t58);
    res[13] = (0.5*t61 + 0.5*n[1]*t70);
    res[14] = (0.025*t62 + 0.025*t65);
    res[15] = (0.017857142857142856*t66 + 0.017857142857142856*t69);
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
    T t2 = std::sqrt((((Q[3]*n[0] + Q[6]*n[1])*(Q[3]*n[0] + Q[6]*n[1])) + 0.6*((Q[4]*n[0] + Q[7]*n[1])*(Q[4]*n[0] + Q[7]*n[1])) + (p[0]*std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1]))/(t0*t0))));
    T t3 = (Q[2]*n[0] + Q[5]*n[1]);
    SimpleArray<T, 1> res;
    res[0] = std::max(t1*std::fabs((t2 + t3)), t1*std::fabs((t2 - t3)));
    return res;
    }

};
