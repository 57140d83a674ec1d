#pragma once
// Generated by models/gen_sme.py (sme2d_l4: dim=2 level=4). Do not edit by hand.
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
    static constexpr int n_dof_q = 12;
    PORTABLE_FN static inline SimpleArray<T, 12> numerical_flux(
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
    T t14 = Q_minus[10]*Q_minus[5];
    T t15 = Q_minus[11]*Q_minus[6];
    T t16 = 105.0*Q_minus[8];
    T t17 = Q_minus[4]*Q_minus[9];
    T t18 = t13*(35.0*t15 + 45.0*t14 + 63.0*t17 + Q_minus[3]*t16 + 315.0*Q_minus[2]*Q_minus[7]);
    T t19 = (1.0/((t5*t5)*std::sqrt(((t7*t7*t7*t7) + (std::max((T)1e-12, t6)*std::max((T)1e-12, t6)*std::max((T)1e-12, t6)*std::max((T)1e-12, t6))))));
    T t20 = t19*(t7*t7*t7);
    T t21 = n[1]*t20;
    T t22 = 2.0*t21;
    T t23 = Q_plus[10]*Q_plus[5];
    T t24 = Q_plus[11]*Q_plus[6];
    T t25 = 105.0*Q_plus[8];
    T t26 = Q_plus[4]*Q_plus[9];
    T t27 = t13*(35.0*t24 + 45.0*t23 + 63.0*t26 + Q_plus[3]*t25 + 315.0*Q_plus[2]*Q_plus[7]);
    T t28 = (t3*t3);
    T t29 = 315.0*p[0];
    T t30 = t3*t9;
    T t31 = t13*t30;
    T t32 = 630.0*t31;
    T t33 = (Q_minus[3]*Q_minus[3]);
    T t34 = 210.0*t31;
    T t35 = (Q_minus[4]*Q_minus[4]);
    T t36 = 126.0*t31;
    T t37 = (Q_minus[5]*Q_minus[5]);
    T t38 = 90.0*t31;
    T t39 = (Q_minus[6]*Q_minus[6]);
    T t40 = 70.0*t13;
    T t41 = t30*t40;
    T t42 = (t7*t7);
    T t43 = t19*t7;
    T t44 = t13*t43;
    T t45 = 630.0*t44;
    T t46 = (Q_plus[3]*Q_plus[3]);
    T t47 = 210.0*t44;
    T t48 = (Q_plus[4]*Q_plus[4]);
    T t49 = 126.0*t44;
    T t50 = (Q_plus[5]*Q_plus[5]);
    T t51 = 90.0*t44;
    T t52 = (Q_plus[6]*Q_plus[6]);
    T t53 = t40*t43;
    T t54 = 105.0*Q_minus[3];
    T t55 = 42.0*Q_minus[3];
    T t56 = 27.0*Q_minus[4];
    T t57 = 20.0*Q_minus[6];
    T t58 = n[0]*t10;
    T t59 = 2.0*t58;
    T t60 = 105.0*Q_plus[3];
    T t61 = 42.0*Q_plus[3];
    T t62 = 27.0*Q_plus[4];
    T t63 = 20.0*Q_plus[6];
    T t64 = n[0]*t20;
    T t65 = 2.0*t64;
    T t66 = Q_minus[11]*Q_minus[5];
    T t67 = Q_minus[4]*Q_minus[8];
    T t68 = Q_minus[5]*Q_minus[9];
    T t69 = (20.0*t66 + 27.0*t68 + 42.0*t67 + Q_minus[10]*t56 + Q_minus[10]*t57 + Q_minus[2]*t16 + Q_minus[7]*t54 + Q_minus[9]*t55);
    T t70 = Q_plus[11]*Q_plus[5];
    T t71 = Q_plus[4]*Q_plus[8];
    T t72 = Q_plus[5]*Q_plus[9];
    T t73 = (20.0*t70 + 27.0*t72 + 42.0*t71 + Q_plus[10]*t62 + Q_plus[10]*t63 + Q_plus[2]*t25 + Q_plus[7]*t60 + Q_plus[9]*t61);
    T t74 = 0.004761904761904762*t13;
    T t75 = 693.0*Q_minus[2];
    T t76 = 297.0*Q_minus[3];
    T t77 = 198.0*Q_minus[4];
    T t78 = 693.0*Q_plus[2];
    T t79 = 297.0*Q_plus[3];
    T t80 = 198.0*Q_plus[4];
    T t81 = 693.0*Q_minus[7];
    T t82 = Q_minus[5]*Q_minus[8];
    T t83 = Q_minus[6]*Q_minus[9];
    T t84 = (100.0*t15 + 132.0*t14 + 198.0*t17 + 198.0*t83 + 297.0*t82 + Q_minus[10]*t76 + Q_minus[11]*t77 + Q_minus[4]*t81 + Q_minus[9]*t75 + 462.0*Q_minus[3]*Q_minus[8]);
    T t85 = 693.0*Q_plus[7];
    T t86 = Q_plus[5]*Q_plus[8];
    T t87 = Q_plus[6]*Q_plus[9];
    T t88 = (100.0*t24 + 132.0*t23 + 198.0*t26 + 198.0*t87 + 297.0*t86 + Q_plus[10]*t79 + Q_plus[11]*t80 + Q_plus[4]*t85 + Q_plus[9]*t78 + 462.0*Q_plus[3]*Q_plus[8]);
    T t89 = 0.0007215007215007215*t13;
    T t90 = 495.0*Q_minus[2];
    T t91 = 220.0*Q_minus[3];
    T t92 = 132.0*Q_minus[4];
    T t93 = 90.0*Q_minus[6];
    T t94 = 495.0*Q_plus[2];
    T t95 = 220.0*Q_plus[3];
    T t96 = 132.0*Q_plus[4];
    T t97 = 90.0*Q_plus[6];
    T t98 = 495.0*Q_minus[7];
    T t99 = 220.0*Q_minus[8];
    T t100 = (90.0*t66 + 132.0*t68 + 297.0*t67 + Q_minus[10]*t90 + Q_minus[10]*t92 + Q_minus[10]*t93 + Q_minus[11]*t91 + Q_minus[5]*t98 + Q_minus[6]*t99 + Q_minus[9]*t76);
    T t101 = 495.0*Q_plus[7];
    T t102 = 220.0*Q_plus[8];
    T t103 = (90.0*t70 + 132.0*t72 + 297.0*t71 + Q_plus[10]*t94 + Q_plus[10]*t96 + Q_plus[10]*t97 + Q_plus[11]*t95 + Q_plus[5]*t101 + Q_plus[6]*t102 + Q_plus[9]*t79);
    T t104 = 0.00101010101010101*t13;
    T t105 = 5005.0*Q_minus[2];
    T t106 = 2860.0*Q_minus[3];
    T t107 = 1300.0*Q_minus[4];
    T t108 = 5005.0*Q_plus[2];
    T t109 = 2860.0*Q_plus[3];
    T t110 = 1300.0*Q_plus[4];
    T t111 = 5005.0*Q_minus[7];
    T t112 = (810.0*t15 + 1170.0*t14 + 1300.0*t83 + 2574.0*t17 + 2860.0*t82 + Q_minus[10]*t106 + Q_minus[11]*t105 + Q_minus[11]*t107 + Q_minus[6]*t111);
    T t113 = 5005.0*Q_plus[7];
    T t114 = (810.0*t24 + 1170.0*t23 + 1300.0*t87 + 2574.0*t26 + 2860.0*t86 + Q_plus[10]*t109 + Q_plus[11]*t108 + Q_plus[11]*t110 + Q_plus[6]*t113);
    T t115 = 9.99000999000999e-05*t13;
    T t116 = (Q_minus[10]*Q_minus[10]);
    T t117 = (Q_minus[11]*Q_minus[11]);
    T t118 = (Q_minus[8]*Q_minus[8]);
    T t119 = (Q_minus[9]*Q_minus[9]);
    T t120 = (Q_plus[10]*Q_plus[10]);
    T t121 = (Q_plus[11]*Q_plus[11]);
    T t122 = (Q_plus[8]*Q_plus[8]);
    T t123 = (Q_plus[9]*Q_plus[9]);
    T t124 = Q_minus[10]*Q_minus[11];
    T t125 = Q_minus[10]*Q_minus[9];
    T t126 = Q_minus[8]*Q_minus[9];
    T t127 = Q_plus[10]*Q_plus[11];
    T t128 = Q_plus[10]*Q_plus[9];
    T t129 = Q_plus[8]*Q_plus[9];
    T t130 = Q_minus[10]*Q_minus[8];
    T t131 = Q_minus[11]*Q_minus[9];
    T t132 = Q_plus[10]*Q_plus[8];
    T t133 = Q_plus[11]*Q_plus[9];
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = (0.5*Q_minus[2]*n[0]*t4 + 0.5*Q_minus[7]*n[1]*t4 + 0.5*Q_plus[2]*n[0]*t8 + 0.5*Q_plus[7]*n[1]*t8);
    res[2] = (0.0007936507936507937*t12*t18 + 0.0007936507936507937*t22*t27 + 0.0007936507936507937*n[0]*t28*(t29 + t32*(Q_minus[2]*Q_minus[2]) + t33*t34 + t35*t36 + t37*t38 + t39*t41) + 0.0007936507936507937*n[0]*t42*(t29 + t45*(Q_plus[2]*Q_plus[2]) + t46*t47 + t48*t49 + t50*t51 + t52*t53));
    res[3] = t74*(t11*t69 + t21*t73 + t59*(Q_minus[2]*t54 + Q_minus[4]*t55 + Q_minus[5]*t56 + Q_minus[5]*t57) + t65*(Q_plus[2]*t60 + Q_plus[4]*t61 + Q_plus[5]*t62 + Q_plus[5]*t63));
    res[4] = t89*(t11*t84 + t21*t88 + t59*(50.0*t39 + 66.0*t37 + 99.0*t35 + 231.0*t33 + Q_minus[4]*t75 + Q_minus[5]*t76 + Q_minus[6]*t77) + t65*(50.0*t52 + 66.0*t50 + 99.0*t48 + 231.0*t46 + Q_plus[4]*t78 + Q_plus[5]*t79 + Q_plus[6]*t80));
    res[5] = t104*(t100*t11 + t103*t21 + t59*(Q_minus[4]*t76 + Q_minus[5]*t90 + Q_minus[5]*t92 + Q_minus[5]*t93 + Q_minus[6]*t91) + t65*(Q_plus[4]*t79 + Q_plus[5]*t94 + Q_plus[5]*t96 + Q_plus[5]*t97 + Q_plus[6]*t95));
    res[6] = t115*(t11*t112 + t114*t21 + t59*(405.0*t39 + 585.0*t37 + 1287.0*t35 + Q_minus[5]*t106 + Q_minus[6]*t105 + Q_minus[6]*t107) + t65*(405.0*t52 + 585.0*t50 + 1287.0*t48 + Q_plus[5]*t109 + Q_plus[6]*t108 + Q_plus[6]*t110));
    res[7] = (0.0007936507936507937*t18*t59 + 0.0007936507936507937*t27*t65 + 0.0007936507936507937*n[1]*t28*(t29 + t116*t38 + t117*t41 + t118*t34 + t119*t36 + t32*(Q_minus[7]*Q_minus[7])) + 0.0007936507936507937*n[1]*t42*(t29 + t120*t51 + t121*t53 + t122*t47 + t123*t49 + t45*(Q_plus[7]*Q_plus[7])));
    res[8] = t74*(t12*(20.0*t124 + 27.0*t125 + 42.0*t126 + Q_minus[7]*t16) + t22*(20.0*t127 + 27.0*t128 + 42.0*t129 + Q_plus[7]*t25) + t58*t69 + t64*t73);
    res[9] = t89*(t12*(50.0*t117 + 66.0*t116 + 99.0*t119 + 198.0*t131 + 231.0*t118 + 297.0*t130 + Q_minus[9]*t81) + t22*(50.0*t121 + 66.0*t120 + 99.0*t123 + 198.0*t133 + 231.0*t122 + 297.0*t132 + Q_plus[9]*t85) + t58*t84 + t64*t88);
    res[10] = t104*(t100*t58 + t103*t64 + t12*(90.0*t124 + 132.0*t125 + 297.0*t126 + Q_minus[10]*t98 + Q_minus[11]*t99) + t22*(90.0*t127 + 132.0*t128 + 297.0*t129 + Q_plus[10]*t101 + Q_plus[11]*t102));
    res[11] = t115*(t112*t58 + t114*t64 + t12*(405.0*t117 + 585.0*t116 + 1287.0*t119 + 1300.0*t131 + 2860.0*t130 + Q_minus[11]*t111) + t22*(405.0*t121 + 585.0*t120 + 1287.0*t123 + 1300.0*t133 + 2860.0*t132 + Q_plus[11]*t113));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 24> numerical_fluctuations(
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
    T t7 = t6*(Q_minus[2]*n[0] + Q_minus[7]*n[1]);
    T t8 = (1.0/(t5*t5));
    T t9 = std::max((T)1e-14, t1);
    T t10 = std::sqrt((t8*((Q_minus[3]*n[0] + Q_minus[8]*n[1])*(Q_minus[3]*n[0] + Q_minus[8]*n[1])) + 0.3333333333333333*t8*((Q_minus[11]*n[1] + Q_minus[6]*n[0])*(Q_minus[11]*n[1] + Q_minus[6]*n[0])) + 0.6*t8*((Q_minus[4]*n[0] + Q_minus[9]*n[1])*(Q_minus[4]*n[0] + Q_minus[9]*n[1])) + 0.42857142857142855*t8*((Q_minus[10]*n[1] + Q_minus[5]*n[0])*(Q_minus[10]*n[1] + Q_minus[5]*n[0])) + (p[0]*(t2*t2*t2)/(t9*t9))));
    T t11 = (t2/(t9));
    T t12 = std::max((T)1e-14, Q_plus[1]);
    T t13 = (1.0/(t12));
    T t14 = t13*(Q_plus[2]*n[0] + Q_plus[7]*n[1]);
    T t15 = (1.0/(t12*t12));
    T t16 = std::max((T)1e-14, t3);
    T t17 = std::sqrt((t15*((Q_plus[3]*n[0] + Q_plus[8]*n[1])*(Q_plus[3]*n[0] + Q_plus[8]*n[1])) + 0.3333333333333333*t15*((Q_plus[11]*n[1] + Q_plus[6]*n[0])*(Q_plus[11]*n[1] + Q_plus[6]*n[0])) + 0.6*t15*((Q_plus[4]*n[0] + Q_plus[9]*n[1])*(Q_plus[4]*n[0] + Q_plus[9]*n[1])) + 0.42857142857142855*t15*((Q_plus[10]*n[1] + Q_plus[5]*n[0])*(Q_plus[10]*n[1] + Q_plus[5]*n[0])) + (p[0]*(t4*t4*t4)/(t16*t16))));
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
    T t30 = 420.0*t19;
    T t31 = t29*t30;
    T t32 = Q_minus[4]*t22;
    T t33 = Q_minus[6]*t22;
    T t34 = 5.0*t33;
    T t35 = Q_plus[4]*t24;
    T t36 = Q_plus[6]*t24;
    T t37 = 5.0*t36;
    T t38 = std::sqrt(2.0);
    T t39 = (t2 + t4);
    T t40 = (1.0/std::sqrt(((std::max((T)1e-12, 0.5*t39)*std::max((T)1e-12, 0.5*t39)*std::max((T)1e-12, 0.5*t39)*std::max((T)1e-12, 0.5*t39)) + 0.0625*(t39*t39*t39*t39))));
    T t41 = t38*t39*t40;
    T t42 = t41*((-t34) - t37 + 9.0*t32 + 9.0*t35);
    T t43 = Q_minus[5]*t22;
    T t44 = Q_plus[5]*t24;
    T t45 = (t43 - t44);
    T t46 = n[0]*t45;
    T t47 = Q_minus[10]*t22;
    T t48 = Q_plus[10]*t24;
    T t49 = (t47 - t48);
    T t50 = n[1]*t49;
    T t51 = 3.0*t43;
    T t52 = 3.0*t44;
    T t53 = ((-t51) - t52 + 7.0*t27 + 7.0*t28);
    T t54 = 3.0*t53;
    T t55 = (-t35);
    T t56 = (t32 + t55);
    T t57 = n[0]*t41;
    T t58 = t56*t57;
    T t59 = Q_minus[9]*t22;
    T t60 = Q_plus[9]*t24;
    T t61 = (-t60);
    T t62 = (t59 + t61);
    T t63 = n[1]*t41;
    T t64 = t62*t63;
    T t65 = (t33 - t36);
    T t66 = n[0]*t65;
    T t67 = (t43 + t44);
    T t68 = 5.0*t41;
    T t69 = t67*t68;
    T t70 = Q_minus[11]*t22;
    T t71 = Q_plus[11]*t24;
    T t72 = (t70 - t71);
    T t73 = n[1]*t72;
    T t74 = ((-21.0*t32) + 21.0*t55 + 105.0*t23 + 105.0*t25);
    T t75 = t29*t57;
    T t76 = Q_minus[8]*t22;
    T t77 = Q_plus[8]*t24;
    T t78 = (t76 - t77);
    T t79 = t63*t78;
    T t80 = (t42*t46 + t42*t50 + t54*t58 + t54*t64 + t66*t69 + t69*t73 + t74*t75 + t74*t79);
    T t81 = 924.0*t19;
    T t82 = t56*t81;
    T t83 = (t34 + t37 + 33.0*t32 + 33.0*t35);
    T t84 = t41*t83;
    T t85 = ((-44.0*t33) - 44.0*t36 + 33.0*t32 + 33.0*t35 + 231.0*t23 + 231.0*t25);
    T t86 = t41*t46;
    T t87 = (t67 + 6.0*t27 + 6.0*t28);
    T t88 = 11.0*t87;
    T t89 = t41*t50;
    T t90 = 33.0*t53;
    T t91 = (t58*t85 + t64*t85 + t66*t84 + t73*t84 + t75*t90 + t79*t90 + t86*t88 + t88*t89);
    T t92 = 660.0*t19;
    T t93 = t45*t92;
    T t94 = t41*(t83 + 165.0*t23 + 165.0*t25);
    T t95 = (t51 + t52 + 11.0*t27 + 11.0*t28);
    T t96 = t68*t95;
    T t97 = 22.0*t42;
    T t98 = n[0]*t29;
    T t99 = 22.0*t87;
    T t100 = n[1]*t78;
    T t101 = (t100*t97 + t46*t94 + t50*t94 + t58*t99 + t64*t99 + t66*t96 + t73*t96 + t97*t98);
    T t102 = 4004.0*t19;
    T t103 = t102*t65;
    T t104 = t41*(81.0*t33 + 81.0*t36 + 221.0*t32 + 221.0*t35 + 1001.0*t23 + 1001.0*t25);
    T t105 = 26.0*t84;
    T t106 = n[0]*t56;
    T t107 = n[1]*t62;
    T t108 = 65.0*t95;
    T t109 = 1430.0*t67;
    T t110 = (t104*t66 + t104*t73 + t105*t106 + t105*t107 + t108*t86 + t108*t89 + t109*t75 + t109*t79);
    T t111 = Q_minus[7]*t22;
    T t112 = Q_plus[7]*t24;
    T t113 = t19*(t111 - t112);
    T t114 = (t47 + t48);
    T t115 = (5.0*t70 + 5.0*t71);
    T t116 = t41*(t115 - 9.0*t59 - 9.0*t60);
    T t117 = t116*t46;
    T t118 = t116*t50;
    T t119 = (t61 - t59 + 5.0*t111 + 5.0*t112);
    T t120 = (3.0*t47 + 3.0*t48);
    T t121 = (t120 - 7.0*t76 - 7.0*t77);
    T t122 = 3.0*t121;
    T t123 = t122*t58;
    T t124 = t122*t64;
    T t125 = t30*t78;
    T t126 = t62*t81;
    T t127 = (t115 + 33.0*t59 + 33.0*t60);
    T t128 = t127*t41;
    T t129 = 33.0*t121;
    T t130 = ((-44.0*t70) - 44.0*t71 + 33.0*t59 + 33.0*t60 + 231.0*t111 + 231.0*t112);
    T t131 = (t114 + 6.0*t76 + 6.0*t77);
    T t132 = 11.0*t131;
    T t133 = (t128*t66 + t128*t73 + t130*t58 + t130*t64 + t132*t86 + t132*t89 - t129*t75 - t129*t79);
    T t134 = t49*t92;
    T t135 = t41*(t127 + 165.0*t111 + 165.0*t112);
    T t136 = 22.0*t116;
    T t137 = (t120 + 11.0*t76 + 11.0*t77);
    T t138 = t137*t68;
    T t139 = 22.0*t131;
    T t140 = (t135*t46 + t135*t50 + t138*t66 + t138*t73 + t139*t58 + t139*t64 - t100*t136 - t136*t98);
    T t141 = t102*t72;
    T t142 = t41*(81.0*t70 + 81.0*t71 + 221.0*t59 + 221.0*t60 + 1001.0*t111 + 1001.0*t112);
    T t143 = 26.0*t128;
    T t144 = 65.0*t137;
    T t145 = 1430.0*t114;
    T t146 = (t106*t143 + t107*t143 + t142*t66 + t142*t73 + t144*t86 + t144*t89 + t145*t75 + t145*t79);
    T t147 = p[0]*((Q_minus[1]*Q_minus[1]) - (t2*t2));
    T t148 = t114*t68;
    T t149 = 21.0*t119;
    SimpleArray<T, 24> res;
    res[0] = 0.0;
    res[1] = (-t20);
    res[2] = ((-0.5*t26) - 0.5*n[0]*t21);
    res[3] = ((-0.0011904761904761906*t31) + 0.0011904761904761906*t80);
    res[4] = ((-0.0005411255411255411*t82) + 0.0005411255411255411*t91);
    res[5] = ((-0.0007575757575757576*t93) + 0.0007575757575757576*t101);
    res[6] = ((-0.00012487512487512488*t103) + 0.00012487512487512488*t110);
    res[7] = ((-0.5*t113) - 0.5*n[1]*t21);
    res[8] = ((-0.0011904761904761906*t117) - 0.0011904761904761906*t118 - 0.0011904761904761906*t123 - 0.0011904761904761906*t124 - 0.0011904761904761906*t125 + 0.025*n[0]*t119*t29*t38*t39*t40 + 0.025*n[1]*t119*t38*t39*t40*t78 + 0.005952380952380952*n[0]*t114*t38*t39*t40*t65 + 0.005952380952380952*n[1]*t114*t38*t39*t40*t72);
    res[9] = ((-0.0005411255411255411*t126) + 0.0005411255411255411*t133);
    res[10] = ((-0.0007575757575757576*t134) + 0.0007575757575757576*t140);
    res[11] = ((-0.00012487512487512488*t141) + 0.00012487512487512488*t146);
    res[12] = 0.0;
    res[13] = t20;
    res[14] = (0.5*t26 + 0.5*n[0]*t147);
    res[15] = (0.0011904761904761906*t31 + 0.0011904761904761906*t80);
    res[16] = (0.0005411255411255411*t82 + 0.0005411255411255411*t91);
    res[17] = (0.0007575757575757576*t101 + 0.0007575757575757576*t93);
    res[18] = (0.00012487512487512488*t103 + 0.00012487512487512488*t110);
    res[19] = (0.5*t113 + 0.5*n[1]*t147);
    res[20] = ((-0.0011904761904761906*t117) - 0.0011904761904761906*t118 - 0.0011904761904761906*t123 - 0.0011904761904761906*t124 + 0.0011904761904761906*t125 + 0.0011904761904761906*t148*t66 + 0.0011904761904761906*t148*t73 + 0.0011904761904761906*t149*t75 + 0.0011904761904761906*t149*t79);
    res[21] = (0.0005411255411255411*t126 + 0.0005411255411255411*t133);
    res[22] = (0.0007575757575757576*t134 + 0.0007575757575757576*t140);
    res[23] = (0.00012487512487512488*t141 + 0.00012487512487512488*t146);
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
    T t2 = std::sqrt((((Q[3]*n[0] + Q[8]*n[1])*(Q[3]*n[0] + Q[8]*n[1])) + 0.3333333333333333*((Q[11]*n[1] + Q[6]*n[0])*(Q[11]*n[1] + Q[6]*n[0])) + 0.6*((Q[4]*n[0] + Q[9]*n[1])*(Q[4]*n[0] + Q[9]*n[1])) + 0.42857142857142855*((Q[10]*n[1] + Q[5]*n[0])*(Q[10]*n[1] + Q[5]*n[0])) + (p[0]*std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1]))/(t0*t0))));
    T t3 = (Q[2]*n[0] + Q[7]*n[1]);
    SimpleArray<T, 1> res;
    res[0] = std::max(t1*std::fabs((t2 + t3)), t1*std::fabs((t2 - t3)));
    return res;
    }

};
