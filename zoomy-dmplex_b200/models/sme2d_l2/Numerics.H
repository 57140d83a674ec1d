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
    T t7 = Q_minus[5]*n[1];
    T t8 = Q_plus[2]*n[0];
    T t9 = std::max((T)1e-14, Q_plus[1]);
    T t10 = (1.0/(t9));
    T t11 = (Q_plus[0] + Q_plus[1] + t3);
    T t12 = std::max((T)0.0, t11);
    T t13 = t10*t12;
    T t14 = Q_plus[5]*n[1];
    T t15 = (t5*t5*t5);
    T t16 = (1.0/(t1*t1));
    T t17 = (t16/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)))));
    T t18 = t15*t17;
    T t19 = n[1]*t18;
    T t20 = 2.0*t19;
    T t21 = std::sqrt(2.0);
    T t22 = Q_minus[3]*Q_minus[6];
    T t23 = Q_minus[4]*Q_minus[7];
    T t24 = t21*(3.0*t23 + 5.0*t22 + 15.0*Q_minus[2]*Q_minus[5]);
    T t25 = (t12*t12*t12);
    T t26 = (1.0/(t9*t9));
    T t27 = (t26/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)))));
    T t28 = t25*t27;
    T t29 = n[1]*t28;
    T t30 = 2.0*t29;
    T t31 = Q_plus[3]*Q_plus[6];
    T t32 = Q_plus[4]*Q_plus[7];
    T t33 = t21*(3.0*t32 + 5.0*t31 + 15.0*Q_plus[2]*Q_plus[5]);
    T t34 = (t5*t5);
    T t35 = 15.0*p[0];
    T t36 = t17*t5;
    T t37 = t21*t36;
    T t38 = 30.0*t37;
    T t39 = (Q_minus[3]*Q_minus[3]);
    T t40 = 10.0*t37;
    T t41 = (Q_minus[4]*Q_minus[4]);
    T t42 = 6.0*t21;
    T t43 = t36*t42;
    T t44 = (t12*t12);
    T t45 = t12*t27;
    T t46 = t21*t45;
    T t47 = 30.0*t46;
    T t48 = (Q_plus[3]*Q_plus[3]);
    T t49 = 10.0*t46;
    T t50 = (Q_plus[4]*Q_plus[4]);
    T t51 = t42*t45;
    T t52 = 5.0*Q_minus[2];
    T t53 = 2.0*Q_minus[4];
    T t54 = Q_minus[3]*n[0];
    T t55 = 2.0*t18;
    T t56 = 5.0*Q_plus[2];
    T t57 = 2.0*Q_plus[4];
    T t58 = Q_plus[3]*n[0];
    T t59 = 2.0*t28;
    T t60 = 5.0*Q_minus[5];
    T t61 = 2.0*Q_minus[7];
    T t62 = (Q_minus[3]*t60 + Q_minus[3]*t61 + Q_minus[6]*t52 + Q_minus[6]*t53);
    T t63 = 5.0*Q_plus[5];
    T t64 = 2.0*Q_plus[7];
    T t65 = (Q_plus[3]*t63 + Q_plus[3]*t64 + Q_plus[6]*t56 + Q_plus[6]*t57);
    T t66 = 0.1*t21;
    T t67 = 21.0*Q_minus[2];
    T t68 = n[0]*t18;
    T t69 = 2.0*t68;
    T t70 = 21.0*Q_plus[2];
    T t71 = n[0]*t28;
    T t72 = 2.0*t71;
    T t73 = 21.0*Q_minus[5];
    T t74 = (6.0*t23 + 14.0*t22 + Q_minus[4]*t73 + Q_minus[7]*t67);
    T t75 = 21.0*Q_plus[5];
    T t76 = (6.0*t32 + 14.0*t31 + Q_plus[4]*t75 + Q_plus[7]*t70);
    T t77 = 0.023809523809523808*t21;
    T t78 = (Q_minus[6]*Q_minus[6]);
    T t79 = (Q_minus[7]*Q_minus[7]);
    T t80 = (Q_plus[6]*Q_plus[6]);
    T t81 = (Q_plus[7]*Q_plus[7]);
    T t82 = Q_minus[6]*n[1];
    T t83 = Q_plus[6]*n[1];
    T t84 = t2*(t0 + t7);
    T t85 = std::max((T)1e-14, t4);
    T t86 = std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))));
    T t87 = (t5/(t85));
    T t88 = t10*(t14 + t8);
    T t89 = std::max((T)1e-14, t11);
    T t90 = std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))));
    T t91 = (t12/(t89));
    T t92 = std::max(t87*std::fabs((t84 + t86)), std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))));
    T t93 = 0.5*t92*(t5 - t12);
    T t94 = p[0]*((Q_plus[1]*Q_plus[1]) - t44);
    T t95 = Q_minus[2]*t6;
    T t96 = Q_plus[2]*t13;
    T t97 = t92*(t95 - t96);
    T t98 = Q_minus[3]*t6;
    T t99 = Q_plus[3]*t13;
    T t100 = (t98 - t99);
    T t101 = 20.0*t92;
    T t102 = t100*t101;
    T t103 = (t98 + t99);
    T t104 = Q_minus[4]*t6;
    T t105 = Q_plus[4]*t13;
    T t106 = (-t105);
    T t107 = (t104 + t106);
    T t108 = (t12 + t5);
    T t109 = (t108*t21/std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108))));
    T t110 = n[0]*t109;
    T t111 = t107*t110;
    T t112 = (t106 - t104 + t13*t56 + t52*t6);
    T t113 = t100*t110;
    T t114 = Q_minus[7]*t6;
    T t115 = Q_plus[7]*t13;
    T t116 = (-t115);
    T t117 = (t114 + t116);
    T t118 = n[1]*t109;
    T t119 = t117*t118;
    T t120 = Q_minus[6]*t6;
    T t121 = Q_plus[6]*t13;
    T t122 = (t120 - t121);
    T t123 = t118*t122;
    T t124 = (t103*t111 + t103*t119 + t112*t113 + t112*t123);
    T t125 = 28.0*t92;
    T t126 = t107*t125;
    T t127 = (t104 + t105 + 7.0*t95 + 7.0*t96);
    T t128 = 7.0*t103;
    T t129 = (t111*t127 + t113*t128 + t119*t127 + t123*t128);
    T t130 = Q_minus[5]*t6;
    T t131 = Q_plus[5]*t13;
    T t132 = t92*(t130 - t131);
    T t133 = t101*t122;
    T t134 = (t116 - t114 + t13*t63 + t6*t60);
    T t135 = (t120 + t121);
    T t136 = (t111*t135 + t113*t134 + t119*t135 + t123*t134);
    T t137 = t117*t125;
    T t138 = (t114 + t115 + 7.0*t130 + 7.0*t131);
    T t139 = 7.0*t135;
    T t140 = (t111*t138 + t113*t139 + t119*t138 + t123*t139);
    T t141 = p[0]*((Q_minus[1]*Q_minus[1]) - t34);
    T a_t141 = (0.5*n[0]*w[18] + 0.5*n[1]*w[21]);
    T a_t140 = (0.017857142857142856*w[15] + 0.017857142857142856*w[23]);
    T a_t139 = (a_t140*t113 + a_t140*t123);
    T a_t138 = (a_t140*t111 + a_t140*t119);
    T a_t137 = ((-0.017857142857142856*w[15]) + 0.017857142857142856*w[23]);
    T a_t136 = (0.025*w[14] + 0.025*w[22]);
    T a_t135 = (7.0*a_t139 + a_t136*t111 + a_t136*t119);
    T a_t134 = (a_t136*t113 + a_t136*t123);
    T a_t133 = ((-0.025*w[14]) + 0.025*w[22]);
    T a_t132 = (0.5*w[21] - 0.5*w[13]);
    T a_t131 = (7.0*a_t138 - a_t132*t92);
    T a_t130 = (7.0*a_t138 + a_t132*t92);
    T a_t129 = (0.017857142857142856*w[12] + 0.017857142857142856*w[20]);
    T a_t128 = (a_t129*t113 + a_t129*t123);
    T a_t127 = (a_t129*t111 + a_t129*t119);
    T a_t126 = ((-0.017857142857142856*w[12]) + 0.017857142857142856*w[20]);
    T a_t125 = (a_t126*t107 + a_t137*t117);
    T a_t124 = (0.025*w[11] + 0.025*w[19]);
    T a_t123 = (a_t124*t112 + a_t129*t128 + a_t136*t134 + a_t140*t139);
    T a_t122 = (a_t123*t118 + a_t133*t101);
    T a_t121 = (a_t135 - a_t122);
    T a_t120 = (a_t122 + a_t135);
    T a_t119 = (a_t124*t103 + a_t129*t127 + a_t136*t135 + a_t140*t138);
    T a_t118 = (a_t119*t117 + a_t123*t122);
    T a_t117 = (a_t119*t118 + a_t137*t125);
    T a_t116 = (a_t117 + a_t134);
    T a_t115 = (a_t138 - a_t116);
    T a_t114 = (a_t117 + a_t138 - a_t134);
    T a_t113 = (a_t124*t112 + a_t129*t128 + a_t136*t134 + a_t140*t139);
    T a_t112 = (a_t124*t113 + a_t124*t123);
    T a_t111 = (a_t124*t103 + a_t129*t127 + a_t136*t135 + a_t140*t138);
    T a_t110 = (a_t111*t107 + a_t113*t100);
    T a_t109 = (a_t110*n[0] + a_t118*n[1]);
    T a_t108 = (0.5*(((T)1e-12 < 0.5*t108) ? (-(4.0*a_t109*t108*t21*(std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108))*(((T)0.0 < std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))) ? (0.5/std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))) : (T)0.0)/(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108))))) : (T)0.0) + (a_t109*t21/std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))) - (0.25*a_t109*t21*(t108*t108*t108*t108)*(((T)0.0 < std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))) ? (0.5/std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))) : (T)0.0)/(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))));
    T a_t107 = (a_t111*t110 + a_t126*t125);
    T a_t106 = (a_t107 + a_t112);
    T a_t105 = (a_t127 - a_t106);
    T a_t104 = (a_t107 + a_t127 - a_t112);
    T a_t103 = (7.0*a_t128 + a_t124*t111 + a_t124*t119);
    T a_t102 = ((-0.025*w[11]) + 0.025*w[19]);
    T a_t101 = (a_t102*t100 + a_t133*t122);
    T a_t100 = (a_t102*t101 + a_t113*t110);
    T a_t99 = (a_t103 - a_t100);
    T a_t98 = (a_t100 + a_t103);
    T a_t97 = (0.5*w[18] - 0.5*w[10]);
    T a_t96 = (7.0*a_t127 - a_t97*t92);
    T a_t95 = (7.0*a_t127 + a_t97*t92);
    T a_t94 = ((-0.5*n[0]*w[10]) - 0.5*n[1]*w[13]);
    T a_t93 = (w[17] - w[9]);
    T a_t92 = (20.0*a_t101 + 28.0*a_t125 + a_t132*(t130 - t131) + a_t93*(0.5*t5 - 0.5*t12) + a_t97*(t95 - t96));
    T a_t91 = (std::fabs((t88 + t90))*((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? (T)0.0 : ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0)) + std::fabs((t88 - t90))*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0) : (T)0.0));
    T a_t90 = ((-(((t88 - t90) < (T)0.0) ? (-t91*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0) : (T)0.0)) : t91*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0) : (T)0.0))) + (((t88 + t90) < (T)0.0) ? (-t91*((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? (T)0.0 : ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0))) : t91*((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? (T)0.0 : ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0))));
    T a_t89 = ((-(a_t91*t12/(t89*t89))) - (2.0*a_t90*p[0]*t25*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0)/(t89*t89*t89)));
    T a_t88 = ((((t88 + t90) < (T)0.0) ? (-t91*((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? (T)0.0 : ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0))) : t91*((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? (T)0.0 : ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0))) + (((t88 - t90) < (T)0.0) ? (-t91*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0) : (T)0.0)) : t91*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0) : (T)0.0)));
    T a_t87 = (std::fabs((t84 + t86))*((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? (T)0.0 : a_t92) + std::fabs((t84 - t86))*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? (T)0.0 : ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0)));
    T a_t86 = ((-(((t84 - t86) < (T)0.0) ? (-t87*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? (T)0.0 : ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0))) : t87*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? (T)0.0 : ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0)))) + (((t84 + t86) < (T)0.0) ? (-t87*((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? (T)0.0 : a_t92)) : t87*((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? (T)0.0 : a_t92)));
    T a_t85 = ((-(a_t87*t5/(t85*t85))) - (2.0*a_t86*p[0]*t15*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0)/(t85*t85*t85)));
    T a_t84 = ((((t84 + t86) < (T)0.0) ? (-t87*((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? (T)0.0 : a_t92)) : t87*((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? (T)0.0 : a_t92)) + (((t84 - t86) < (T)0.0) ? (-t87*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? (T)0.0 : ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0))) : t87*((t87*std::fabs((t84 - t86)) < t91*std::fabs((t88 - t90))) ? (T)0.0 : ((t91*std::fabs((t88 + t90)) < std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90)))) ? ((t87*std::fabs((t84 + t86)) < std::max(t91*std::fabs((t88 + t90)), std::max(t87*std::fabs((t84 - t86)), t91*std::fabs((t88 - t90))))) ? a_t92 : (T)0.0) : (T)0.0))));
    T a_t83 = (t59*t66*w[6]*(t63 + t64) + 2.0*a_t90*t26*(t58 + t83)*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0));
    T a_t82 = (t55*t66*w[6]*(t60 + t61) + 2.0*a_t86*t16*(t54 + t82)*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0));
    T a_t81 = (3.0*t30*t77*w[7] + 0.016666666666666666*n[1]*t44*t51*w[5]);
    T a_t80 = (7.0*t30*t77*w[7] + 0.016666666666666666*n[1]*t44*t49*w[5]);
    T a_t79 = (3.0*t20*t77*w[7] + 0.016666666666666666*n[1]*t34*t43*w[5]);
    T a_t78 = (7.0*t20*t77*w[7] + 0.016666666666666666*n[1]*t34*t40*w[5]);
    T a_t77 = (w[4]*(t19*t74 + t29*t76 + t69*(3.0*t41 + 7.0*t39 + Q_minus[4]*t67) + t72*(3.0*t50 + 7.0*t48 + Q_plus[4]*t70)) + w[7]*(t20*(3.0*t79 + 7.0*t78 + Q_minus[7]*t73) + t30*(3.0*t81 + 7.0*t80 + Q_plus[7]*t75) + t68*t74 + t71*t76));
    T a_t76 = (t29*t77*w[4] + t71*t77*w[7]);
    T a_t75 = (Q_plus[4]*a_t76 + Q_plus[7]*t30*t77*w[7]);
    T a_t74 = (t19*t77*w[4] + t68*t77*w[7]);
    T a_t73 = (Q_minus[4]*a_t74 + Q_minus[7]*t20*t77*w[7]);
    T a_t72 = (0.016666666666666666*t33*w[5] + t77*w[4]*(3.0*t50 + 7.0*t48 + Q_plus[4]*t70));
    T a_t71 = (2.0*a_t72 + t65*t66*w[6] + t76*t77*w[7]);
    T a_t70 = (Q_plus[7]*a_t76 + Q_plus[4]*t72*t77*w[4]);
    T a_t69 = (0.016666666666666666*t24*w[5] + t77*w[4]*(3.0*t41 + 7.0*t39 + Q_minus[4]*t67));
    T a_t68 = (2.0*a_t69 + t62*t66*w[6] + t74*t77*w[7]);
    T a_t67 = (Q_minus[7]*a_t74 + Q_minus[4]*t69*t77*w[4]);
    T a_t66 = (w[3]*(t19*t62 + t29*t65 + t54*t55*(t52 + t53) + t58*t59*(t56 + t57)) + w[6]*(t62*t68 + t65*t71 + t55*t82*(t60 + t61) + t59*t83*(t63 + t64)));
    T a_t65 = (t29*t66*w[3] + t66*t71*w[6]);
    T a_t64 = (Q_plus[3]*a_t65 + t59*t66*t83*w[6]);
    T a_t63 = (Q_plus[3]*a_t65 + a_t134*t13 + t59*t66*t83*w[6]);
    T a_t62 = (t19*t66*w[3] + t66*t68*w[6]);
    T a_t61 = (Q_minus[3]*a_t62 + t55*t66*t82*w[6]);
    T a_t60 = (Q_minus[3]*a_t62 + a_t134*t6 + t55*t66*t82*w[6]);
    T a_t59 = (t58*t66*w[3]*(t56 + t57) + t66*t83*w[6]*(t63 + t64));
    T a_t58 = (t59*t66*w[3]*(t56 + t57) + 2.0*a_t90*t26*(t58 + t83)*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0));
    T a_t57 = (Q_plus[6]*a_t65 + t58*t59*t66*w[3]);
    T a_t56 = (Q_plus[6]*a_t65 + a_t112*t13 + t58*t59*t66*w[3]);
    T a_t55 = (t54*t66*w[3]*(t52 + t53) + t66*t82*w[6]*(t60 + t61));
    T a_t54 = (t55*t66*w[3]*(t52 + t53) + 2.0*a_t86*t16*(t54 + t82)*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0));
    T a_t53 = (Q_minus[6]*a_t62 + t54*t55*t66*w[3]);
    T a_t52 = (Q_minus[6]*a_t62 + a_t112*t6 + t54*t55*t66*w[3]);
    T a_t51 = (0.016666666666666666*n[0]*t44*t50*w[2] + 0.016666666666666666*n[1]*t44*t81*w[5]);
    T a_t50 = (3.0*t72*t77*w[4] + 0.016666666666666666*n[0]*t44*t51*w[2]);
    T a_t49 = (0.016666666666666666*n[0]*t44*t48*w[2] + 0.016666666666666666*n[1]*t44*t80*w[5]);
    T a_t48 = (7.0*t72*t77*w[4] + 0.016666666666666666*n[0]*t44*t49*w[2]);
    T a_t47 = (0.016666666666666666*n[0]*t44*w[2]*(Q_plus[2]*Q_plus[2]) + 0.016666666666666666*n[1]*t44*w[5]*(Q_plus[5]*Q_plus[5]));
    T a_t46 = (10.0*a_t49 + 30.0*a_t47);
    T a_t45 = (a_t46*t21 + a_t51*t42);
    T a_t44 = ((-a_t94*p[0]) + 0.016666666666666666*n[0]*w[2]*(t35 + t47*(Q_plus[2]*Q_plus[2]) + t48*t49 + t50*t51) + 0.016666666666666666*n[1]*w[5]*(t35 + t47*(Q_plus[5]*Q_plus[5]) + t49*t80 + t51*t81));
    T a_t43 = (0.016666666666666666*n[0]*t34*t41*w[2] + 0.016666666666666666*n[1]*t34*t79*w[5]);
    T a_t42 = (a_t43*t36 + a_t51*t45);
    T a_t41 = (3.0*t69*t77*w[4] + 0.016666666666666666*n[0]*t34*t43*w[2]);
    T a_t40 = (0.016666666666666666*n[0]*t34*t39*w[2] + 0.016666666666666666*n[1]*t34*t78*w[5]);
    T a_t39 = (7.0*t69*t77*w[4] + 0.016666666666666666*n[0]*t34*t40*w[2]);
    T a_t38 = (0.016666666666666666*n[0]*t34*w[2]*(Q_minus[2]*Q_minus[2]) + 0.016666666666666666*n[1]*t34*w[5]*(Q_minus[5]*Q_minus[5]));
    T a_t37 = (10.0*a_t40 + 30.0*a_t38);
    T a_t36 = (a_t37*t21 + a_t43*t42);
    T a_t35 = (0.016666666666666666*n[0]*t34*w[2] + 0.016666666666666666*n[0]*t44*w[2] + 0.016666666666666666*n[1]*t34*w[5] + 0.016666666666666666*n[1]*t44*w[5]);
    T a_t34 = ((-a_t141*p[0]) + 0.016666666666666666*n[0]*w[2]*(t35 + t38*(Q_minus[2]*Q_minus[2]) + t39*t40 + t41*t43) + 0.016666666666666666*n[1]*w[5]*(t35 + t38*(Q_minus[5]*Q_minus[5]) + t40*t78 + t43*t79));
    T a_t33 = (0.016666666666666666*t30*w[2] + 0.016666666666666666*t72*w[5]);
    T a_t32 = (6.0*a_t76 + 3.0*a_t33*t21);
    T a_t31 = (14.0*a_t76 + 5.0*a_t33*t21);
    T a_t30 = (0.016666666666666666*t33*w[2] + t77*w[7]*(3.0*t81 + 7.0*t80 + Q_plus[7]*t75));
    T a_t29 = (2.0*a_t30 + t65*t66*w[3] + t76*t77*w[4]);
    T a_t28 = (2.0*a_t59 + a_t29*n[1] + a_t71*n[0]);
    T a_t27 = (a_t28*t25 + a_t45*t12);
    T a_t26 = ((a_t27/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) + a_t90*((t58 + t83)*(t58 + t83))*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0) + 0.6*a_t90*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1]))*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0));
    T a_t25 = (a_t28*t27 + (a_t90*p[0]*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0)/(t89*t89)));
    T a_t24 = (0.016666666666666666*t20*w[2] + 0.016666666666666666*t69*w[5]);
    T a_t23 = (6.0*a_t74 + 3.0*a_t24*t21);
    T a_t22 = (14.0*a_t74 + 5.0*a_t24*t21);
    T a_t21 = (6.0*a_t42 + 0.1*a_t66 + 0.023809523809523808*a_t77 + a_t24*(3.0*t23 + 5.0*t22 + 15.0*Q_minus[2]*Q_minus[5]) + a_t33*(3.0*t32 + 5.0*t31 + 15.0*Q_plus[2]*Q_plus[5]) + a_t37*t36 + a_t46*t45 + (a_t109*t108/std::sqrt(((std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)*std::max((T)1e-12, 0.5*t108)) + 0.0625*(t108*t108*t108*t108)))));
    T a_t20 = (0.016666666666666666*t24*w[2] + t77*w[7]*(3.0*t79 + 7.0*t78 + Q_minus[7]*t73));
    T a_t19 = (2.0*a_t20 + t62*t66*w[3] + t74*t77*w[4]);
    T a_t18 = (2.0*a_t55 + a_t19*n[1] + a_t68*n[0]);
    T a_t17 = (a_t18*t15 + a_t36*t5);
    T a_t16 = ((a_t17/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) + a_t86*((t54 + t82)*(t54 + t82))*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0) + 0.6*a_t86*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1]))*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0));
    T a_t15 = (a_t18*t17 + (a_t86*p[0]*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0)/(t85*t85)));
    T a_t14 = (a_t88*t10 + 0.5*t13*w[1]);
    T a_t13 = (Q_plus[2]*a_t96 + Q_plus[3]*a_t99 + Q_plus[4]*a_t105 + Q_plus[5]*a_t131 + Q_plus[6]*a_t121 + Q_plus[7]*a_t115 + a_t112*t56 + a_t134*t63 + 0.5*t14*w[1] + 0.5*t8*w[1]);
    T a_t12 = (a_t108 + a_t13*t10 + a_t45*t27 + (a_t91/(t89)) + 2.0*a_t44*t12 + 3.0*a_t25*(t12*t12) - 0.5*a_t93*t92 - (4.0*a_t27*t26*(t12*t12*t12)*(((T)0.0 < std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) ? (0.5/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) : (T)0.0)/(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))));
    T a_t11 = ((((T)0.0 < t11) ? a_t12 : (T)0.0) + (((T)1e-12 < t11) ? (-(4.0*a_t27*t26*(std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))*(((T)0.0 < std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) ? (0.5/std::sqrt(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11))))) : (T)0.0)/(((t12*t12*t12*t12) + (std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)*std::max((T)1e-12, t11)))))) : (T)0.0) + (((T)1e-14 < t11) ? a_t89 : (T)0.0));
    T a_t10 = (a_t13*t12 + a_t88*(t14 + t8));
    T a_t9 = ((-(a_t10/(t9*t9))) - (2.0*a_t26/(t9*t9*t9)));
    T a_t8 = (a_t88*t10 + 0.5*t13*w[1]);
    T a_t7 = (a_t84*t2 + 0.5*t6*w[1]);
    T a_t6 = (Q_minus[2]*a_t95 + Q_minus[3]*a_t98 + Q_minus[4]*a_t104 + Q_minus[5]*a_t130 + Q_minus[6]*a_t120 + Q_minus[7]*a_t114 + a_t112*t52 + a_t134*t60 + 0.5*t0*w[1] + 0.5*t7*w[1]);
    T a_t5 = (a_t108 + a_t36*t17 + a_t6*t2 + (a_t87/(t85)) + 0.5*a_t93*t92 + 2.0*a_t34*t5 + 3.0*a_t15*(t5*t5) - (4.0*a_t17*t16*(t5*t5*t5)*(((T)0.0 < std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) ? (0.5/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) : (T)0.0)/(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))));
    T a_t4 = ((((T)0.0 < t4) ? a_t5 : (T)0.0) + (((T)1e-12 < t4) ? (-(4.0*a_t17*t16*(std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))*(((T)0.0 < std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) ? (0.5/std::sqrt(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4))))) : (T)0.0)/(((t5*t5*t5*t5) + (std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)*std::max((T)1e-12, t4)))))) : (T)0.0) + (((T)1e-14 < t4) ? a_t85 : (T)0.0));
    T a_t3 = (a_t11 + a_t4);
    T a_t2 = (a_t6*t5 + a_t84*(t0 + t7));
    T a_t1 = ((-(a_t2/(t1*t1))) - (2.0*a_t16/(t1*t1*t1)));
    T a_t0 = (a_t84*t2 + 0.5*t6*w[1]);
    g[0] = (a_t4 + ((Q_minus[0] < Q_plus[0]) ? (T)0.0 : (-a_t3)));
    g[1] = (a_t4 + 2.0*Q_minus[1]*a_t141*p[0] + (((T)1e-14 < Q_minus[1]) ? a_t1 : (T)0.0));
    g[2] = (5.0*a_t52 + 21.0*a_t67 + a_t0*n[0] + a_t95*t6 + 15.0*Q_minus[5]*a_t24*t21 + 0.03333333333333333*Q_minus[2]*n[0]*t34*t38*w[2]);
    g[3] = (Q_minus[6]*a_t22 + a_t54*n[0] + a_t62*t60 + a_t62*t61 + a_t98*t6 + 2.0*Q_minus[3]*a_t39);
    g[4] = (2.0*a_t53 + Q_minus[7]*a_t23 + a_t104*t6 + a_t74*t73 + 2.0*Q_minus[4]*a_t41 + t67*t69*t77*w[4] + 1.2*a_t86*n[0]*t16*(Q_minus[4]*n[0] + Q_minus[7]*n[1])*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0));
    g[5] = (5.0*a_t60 + 21.0*a_t73 + a_t130*t6 + a_t7*n[1] + 15.0*Q_minus[2]*a_t24*t21 + 0.03333333333333333*Q_minus[5]*n[1]*t34*t38*w[5]);
    g[6] = (Q_minus[3]*a_t22 + a_t120*t6 + a_t62*t52 + a_t62*t53 + a_t82*n[1] + 2.0*Q_minus[6]*a_t78);
    g[7] = (2.0*a_t61 + Q_minus[4]*a_t23 + a_t114*t6 + a_t74*t67 + 2.0*Q_minus[7]*a_t79 + t20*t73*t77*w[7] + 1.2*a_t86*n[1]*t16*(Q_minus[4]*n[0] + Q_minus[7]*n[1])*(((T)0.0 < std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) ? (0.5/std::sqrt((t16*((t54 + t82)*(t54 + t82)) + 0.6*t16*((Q_minus[4]*n[0] + Q_minus[7]*n[1])*(Q_minus[4]*n[0] + Q_minus[7]*n[1])) + (p[0]*t15/(t85*t85))))) : (T)0.0));
    g[8] = (a_t11 + ((Q_minus[0] < Q_plus[0]) ? (-a_t3) : (T)0.0));
    g[9] = (a_t11 + 2.0*Q_plus[1]*a_t94*p[0] + (((T)1e-14 < Q_plus[1]) ? a_t9 : (T)0.0));
    g[10] = (5.0*a_t56 + 21.0*a_t70 + a_t8*n[0] + a_t96*t13 + 15.0*Q_plus[5]*a_t33*t21 + 0.03333333333333333*Q_plus[2]*n[0]*t44*t47*w[2]);
    g[11] = (Q_plus[6]*a_t31 + a_t58*n[0] + a_t65*t63 + a_t65*t64 + a_t99*t13 + 2.0*Q_plus[3]*a_t48);
    g[12] = (2.0*a_t57 + Q_plus[7]*a_t32 + a_t105*t13 + a_t76*t75 + 2.0*Q_plus[4]*a_t50 + t70*t72*t77*w[4] + 1.2*a_t90*n[0]*t26*(Q_plus[4]*n[0] + Q_plus[7]*n[1])*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0));
    g[13] = (5.0*a_t63 + 21.0*a_t75 + a_t131*t13 + a_t14*n[1] + 15.0*Q_plus[2]*a_t33*t21 + 0.03333333333333333*Q_plus[5]*n[1]*t44*t47*w[5]);
    g[14] = (Q_plus[3]*a_t31 + a_t121*t13 + a_t65*t56 + a_t65*t57 + a_t83*n[1] + 2.0*Q_plus[6]*a_t80);
    g[15] = (2.0*a_t64 + Q_plus[4]*a_t32 + a_t115*t13 + a_t76*t70 + 2.0*Q_plus[7]*a_t81 + t30*t75*t77*w[7] + 1.2*a_t90*n[1]*t26*(Q_plus[4]*n[0] + Q_plus[7]*n[1])*(((T)0.0 < std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) ? (0.5/std::sqrt((t26*((t58 + t83)*(t58 + t83)) + 0.6*t26*((Q_plus[4]*n[0] + Q_plus[7]*n[1])*(Q_plus[4]*n[0] + Q_plus[7]*n[1])) + (p[0]*t25/(t89*t89))))) : (T)0.0));
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
