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

template <typename T>
struct Model {
    static constexpr int n_dof_q    = 12;
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
    PORTABLE_FN static inline SimpleArray<T, 12> flux_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = ((Q[3]*Q[3])/3.0);
    T t1 = (Q[4]*Q[4]);
    T t2 = (Q[5]*Q[5]);
    T t3 = (Q[6]*Q[6]);
    T t4 = Q[3]*Q[4];
    T t5 = Q[4]*Q[5];
    T t6 = Q[5]*Q[6];
    T t7 = 2.0*Qaux[0];
    T t8 = Q[3]*Q[5];
    T t9 = Q[4]*Q[6];
    T t10 = (4.0/9.0)*Q[3];
    T t11 = Q[10]*Q[5];
    T t12 = Q[11]*Q[6];
    T t13 = Q[3]*Q[8];
    T t14 = Q[4]*Q[9];
    T t15 = Q[10]*Q[4];
    T t16 = Q[10]*Q[6];
    T t17 = Q[11]*Q[5];
    T t18 = Q[3]*Q[9];
    T t19 = Q[4]*Q[8];
    T t20 = Q[5]*Q[9];
    T t21 = Q[10]*Q[3];
    T t22 = Q[11]*Q[4];
    T t23 = Q[5]*Q[8];
    T t24 = Q[6]*Q[9];
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*(t0 + (Q[2]*Q[2]) + (t1/5.0) + (t2/7.0) + (t3/9.0));
    res[3] = t7*((2.0/5.0)*t4 + (4.0/21.0)*t6 + (9.0/35.0)*t5 + Q[2]*Q[3]);
    res[4] = t7*(t0 + (t1/7.0) + (2.0/7.0)*t9 + (2.0/21.0)*t2 + (3.0/7.0)*t8 + (50.0/693.0)*t3 + Q[2]*Q[4]);
    res[5] = t7*((2.0/11.0)*t6 + (3.0/5.0)*t4 + (4.0/15.0)*t5 + Q[2]*Q[5] + Q[6]*t10);
    res[6] = t7*((4.0/7.0)*t8 + (9.0/35.0)*t1 + (9.0/77.0)*t2 + (20.0/77.0)*t9 + (81.0/1001.0)*t3 + Q[2]*Q[6]);
    res[7] = Qaux[0]*((t13/3.0) + (t14/5.0) + (t11/7.0) + (t12/9.0) + Q[2]*Q[7]);
    res[8] = Qaux[0]*((2.0/5.0)*t18 + (2.0/5.0)*t19 + (4.0/21.0)*t16 + (4.0/21.0)*t17 + (9.0/35.0)*t15 + (9.0/35.0)*t20 + Q[2]*Q[8] + Q[3]*Q[7]);
    res[9] = Qaux[0]*((2.0/3.0)*t13 + (2.0/7.0)*t14 + (2.0/7.0)*t22 + (2.0/7.0)*t24 + (3.0/7.0)*t21 + (3.0/7.0)*t23 + (4.0/21.0)*t11 + (100.0/693.0)*t12 + Q[2]*Q[9] + Q[4]*Q[7]);
    res[10] = Qaux[0]*((2.0/11.0)*t16 + (2.0/11.0)*t17 + (3.0/5.0)*t18 + (3.0/5.0)*t19 + (4.0/15.0)*t15 + (4.0/15.0)*t20 + Q[10]*Q[2] + Q[11]*t10 + Q[5]*Q[7] + (4.0/9.0)*Q[6]*Q[8]);
    res[11] = Qaux[0]*((4.0/7.0)*t21 + (4.0/7.0)*t23 + (18.0/35.0)*t14 + (18.0/77.0)*t11 + (20.0/77.0)*t22 + (20.0/77.0)*t24 + (162.0/1001.0)*t12 + Q[11]*Q[2] + Q[6]*Q[7]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> flux_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = Q[10]*Q[5];
    T t1 = Q[11]*Q[6];
    T t2 = Q[3]*Q[8];
    T t3 = Q[4]*Q[9];
    T t4 = Q[10]*Q[4];
    T t5 = Q[10]*Q[6];
    T t6 = Q[11]*Q[5];
    T t7 = Q[3]*Q[9];
    T t8 = Q[4]*Q[8];
    T t9 = Q[5]*Q[9];
    T t10 = Q[10]*Q[3];
    T t11 = Q[11]*Q[4];
    T t12 = Q[5]*Q[8];
    T t13 = Q[6]*Q[9];
    T t14 = (4.0/9.0)*Q[11];
    T t15 = (Q[10]*Q[10]);
    T t16 = (Q[11]*Q[11]);
    T t17 = ((Q[8]*Q[8])/3.0);
    T t18 = (Q[9]*Q[9]);
    T t19 = Q[10]*Q[11];
    T t20 = Q[10]*Q[9];
    T t21 = Q[8]*Q[9];
    T t22 = 2.0*Qaux[0];
    T t23 = Q[10]*Q[8];
    T t24 = Q[11]*Q[9];
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = Q[7];
    res[2] = Qaux[0]*((t2/3.0) + (t3/5.0) + (t0/7.0) + (t1/9.0) + Q[2]*Q[7]);
    res[3] = Qaux[0]*((2.0/5.0)*t7 + (2.0/5.0)*t8 + (4.0/21.0)*t5 + (4.0/21.0)*t6 + (9.0/35.0)*t4 + (9.0/35.0)*t9 + Q[2]*Q[8] + Q[3]*Q[7]);
    res[4] = Qaux[0]*((2.0/3.0)*t2 + (2.0/7.0)*t11 + (2.0/7.0)*t13 + (2.0/7.0)*t3 + (3.0/7.0)*t10 + (3.0/7.0)*t12 + (4.0/21.0)*t0 + (100.0/693.0)*t1 + Q[2]*Q[9] + Q[4]*Q[7]);
    res[5] = Qaux[0]*((2.0/11.0)*t5 + (2.0/11.0)*t6 + (3.0/5.0)*t7 + (3.0/5.0)*t8 + (4.0/15.0)*t4 + (4.0/15.0)*t9 + Q[10]*Q[2] + Q[3]*t14 + Q[5]*Q[7] + (4.0/9.0)*Q[6]*Q[8]);
    res[6] = Qaux[0]*((4.0/7.0)*t10 + (4.0/7.0)*t12 + (18.0/35.0)*t3 + (18.0/77.0)*t0 + (20.0/77.0)*t11 + (20.0/77.0)*t13 + (162.0/1001.0)*t1 + Q[11]*Q[2] + Q[6]*Q[7]);
    res[7] = Qaux[0]*(t17 + (Q[7]*Q[7]) + (t18/5.0) + (t15/7.0) + (t16/9.0));
    res[8] = t22*((2.0/5.0)*t21 + (4.0/21.0)*t19 + (9.0/35.0)*t20 + Q[7]*Q[8]);
    res[9] = t22*(t17 + (t18/7.0) + (2.0/7.0)*t24 + (2.0/21.0)*t15 + (3.0/7.0)*t23 + (50.0/693.0)*t16 + Q[7]*Q[9]);
    res[10] = t22*((2.0/11.0)*t19 + (3.0/5.0)*t21 + (4.0/15.0)*t20 + Q[10]*Q[7] + Q[8]*t14);
    res[11] = t22*((4.0/7.0)*t23 + (9.0/35.0)*t18 + (9.0/77.0)*t15 + (20.0/77.0)*t24 + (81.0/1001.0)*t16 + Q[11]*Q[7]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 144> nonconservative_matrix_x(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (Qaux[0]/35.0);
    T t1 = Qaux[0]*((-9.0*Q[4]) + 5.0*Q[6]);
    T t2 = (Qaux[0]/21.0);
    T t3 = (Q[5] + 6.0*Q[3]);
    T t4 = Qaux[0]*(5.0*Q[6] + 33.0*Q[4]);
    T t5 = (2.0/15.0)*Qaux[0];
    T t6 = Qaux[0]*(3.0*Q[5] + 11.0*Q[3]);
    T t7 = (10.0/7.0)*Qaux[0];
    T t8 = 3.0*Q[10];
    T t9 = 5.0*Q[11];
    T t10 = (t9 - 9.0*Q[9]);
    T t11 = (Q[10] + 6.0*Q[8]);
    T t12 = Qaux[0]*(t9 + 33.0*Q[9]);
    T t13 = Qaux[0]*(t8 + 11.0*Q[8]);
    SimpleArray<T, 144> res;
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
    res[23] = 0.0;
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
    res[35] = 0.0;
    res[36] = 0.0;
    res[37] = 0.0;
    res[38] = 0.0;
    res[39] = Qaux[0]*((-Q[2]) + (Q[4]/5.0));
    res[40] = t0*((-7.0*Q[3]) + 3.0*Q[5]);
    res[41] = (t1/105.0);
    res[42] = (-Q[5]*t2);
    res[43] = 0.0;
    res[44] = 0.0;
    res[45] = 0.0;
    res[46] = 0.0;
    res[47] = 0.0;
    res[48] = 0.0;
    res[49] = 0.0;
    res[50] = 0.0;
    res[51] = Qaux[0]*((-Q[3]) + (3.0/7.0)*Q[5]);
    res[52] = Qaux[0]*((-Q[2]) - (Q[4]/7.0) + (4.0/21.0)*Q[6]);
    res[53] = (-t2*t3);
    res[54] = (-(t4/231.0));
    res[55] = 0.0;
    res[56] = 0.0;
    res[57] = 0.0;
    res[58] = 0.0;
    res[59] = 0.0;
    res[60] = 0.0;
    res[61] = 0.0;
    res[62] = 0.0;
    res[63] = (2.0/15.0)*t1;
    res[64] = (-t3*t5);
    res[65] = (-Qaux[0]*(Q[2] + (Q[4]/5.0) + (Q[6]/33.0)));
    res[66] = (-(t6/33.0));
    res[67] = 0.0;
    res[68] = 0.0;
    res[69] = 0.0;
    res[70] = 0.0;
    res[71] = 0.0;
    res[72] = 0.0;
    res[73] = 0.0;
    res[74] = 0.0;
    res[75] = (-Q[5]*t7);
    res[76] = (-(2.0/77.0)*t4);
    res[77] = (-(5.0/77.0)*t6);
    res[78] = (-Qaux[0]*(Q[2] + (17.0/77.0)*Q[4] + (81.0/1001.0)*Q[6]));
    res[79] = 0.0;
    res[80] = 0.0;
    res[81] = 0.0;
    res[82] = 0.0;
    res[83] = 0.0;
    res[84] = 0.0;
    res[85] = 0.0;
    res[86] = 0.0;
    res[87] = 0.0;
    res[88] = 0.0;
    res[89] = 0.0;
    res[90] = 0.0;
    res[91] = 0.0;
    res[92] = 0.0;
    res[93] = 0.0;
    res[94] = 0.0;
    res[95] = 0.0;
    res[96] = 0.0;
    res[97] = 0.0;
    res[98] = 0.0;
    res[99] = Qaux[0]*((-Q[7]) + (Q[9]/5.0));
    res[100] = t0*(t8 - 7.0*Q[8]);
    res[101] = (Qaux[0]*t10/105.0);
    res[102] = (-Q[10]*t2);
    res[103] = 0.0;
    res[104] = 0.0;
    res[105] = 0.0;
    res[106] = 0.0;
    res[107] = 0.0;
    res[108] = 0.0;
    res[109] = 0.0;
    res[110] = 0.0;
    res[111] = Qaux[0]*((-Q[8]) + (3.0/7.0)*Q[10]);
    res[112] = Qaux[0]*((-Q[7]) - (Q[9]/7.0) + (4.0/21.0)*Q[11]);
    res[113] = (-t11*t2);
    res[114] = (-(t12/231.0));
    res[115] = 0.0;
    res[116] = 0.0;
    res[117] = 0.0;
    res[118] = 0.0;
    res[119] = 0.0;
    res[120] = 0.0;
    res[121] = 0.0;
    res[122] = 0.0;
    res[123] = t10*t5;
    res[124] = (-t11*t5);
    res[125] = (-Qaux[0]*(Q[7] + (Q[9]/5.0) + (Q[11]/33.0)));
    res[126] = (-(t13/33.0));
    res[127] = 0.0;
    res[128] = 0.0;
    res[129] = 0.0;
    res[130] = 0.0;
    res[131] = 0.0;
    res[132] = 0.0;
    res[133] = 0.0;
    res[134] = 0.0;
    res[135] = (-Q[10]*t7);
    res[136] = (-(2.0/77.0)*t12);
    res[137] = (-(5.0/77.0)*t13);
    res[138] = (-Qaux[0]*(Q[7] + (17.0/77.0)*Q[9] + (81.0/1001.0)*Q[11]));
    res[139] = 0.0;
    res[140] = 0.0;
    res[141] = 0.0;
    res[142] = 0.0;
    res[143] = 0.0;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 144> nonconservative_matrix_y(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (Qaux[0]/35.0);
    T t1 = Qaux[0]*((-9.0*Q[4]) + 5.0*Q[6]);
    T t2 = (Qaux[0]/21.0);
    T t3 = (Q[5] + 6.0*Q[3]);
    T t4 = Qaux[0]*(5.0*Q[6] + 33.0*Q[4]);
    T t5 = (2.0/15.0)*Qaux[0];
    T t6 = Qaux[0]*(3.0*Q[5] + 11.0*Q[3]);
    T t7 = (10.0/7.0)*Qaux[0];
    T t8 = 3.0*Q[10];
    T t9 = 5.0*Q[11];
    T t10 = (t9 - 9.0*Q[9]);
    T t11 = (Q[10] + 6.0*Q[8]);
    T t12 = Qaux[0]*(t9 + 33.0*Q[9]);
    T t13 = Qaux[0]*(t8 + 11.0*Q[8]);
    SimpleArray<T, 144> res;
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
    res[33] = 0.0;
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
    res[44] = Qaux[0]*((-Q[2]) + (Q[4]/5.0));
    res[45] = t0*((-7.0*Q[3]) + 3.0*Q[5]);
    res[46] = (t1/105.0);
    res[47] = (-Q[5]*t2);
    res[48] = 0.0;
    res[49] = 0.0;
    res[50] = 0.0;
    res[51] = 0.0;
    res[52] = 0.0;
    res[53] = 0.0;
    res[54] = 0.0;
    res[55] = 0.0;
    res[56] = Qaux[0]*((-Q[3]) + (3.0/7.0)*Q[5]);
    res[57] = Qaux[0]*((-Q[2]) - (Q[4]/7.0) + (4.0/21.0)*Q[6]);
    res[58] = (-t2*t3);
    res[59] = (-(t4/231.0));
    res[60] = 0.0;
    res[61] = 0.0;
    res[62] = 0.0;
    res[63] = 0.0;
    res[64] = 0.0;
    res[65] = 0.0;
    res[66] = 0.0;
    res[67] = 0.0;
    res[68] = (2.0/15.0)*t1;
    res[69] = (-t3*t5);
    res[70] = (-Qaux[0]*(Q[2] + (Q[4]/5.0) + (Q[6]/33.0)));
    res[71] = (-(t6/33.0));
    res[72] = 0.0;
    res[73] = 0.0;
    res[74] = 0.0;
    res[75] = 0.0;
    res[76] = 0.0;
    res[77] = 0.0;
    res[78] = 0.0;
    res[79] = 0.0;
    res[80] = (-Q[5]*t7);
    res[81] = (-(2.0/77.0)*t4);
    res[82] = (-(5.0/77.0)*t6);
    res[83] = (-Qaux[0]*(Q[2] + (17.0/77.0)*Q[4] + (81.0/1001.0)*Q[6]));
    res[84] = Q[1]*p[0];
    res[85] = 0.0;
    res[86] = 0.0;
    res[87] = 0.0;
    res[88] = 0.0;
    res[89] = 0.0;
    res[90] = 0.0;
    res[91] = 0.0;
    res[92] = 0.0;
    res[93] = 0.0;
    res[94] = 0.0;
    res[95] = 0.0;
    res[96] = 0.0;
    res[97] = 0.0;
    res[98] = 0.0;
    res[99] = 0.0;
    res[100] = 0.0;
    res[101] = 0.0;
    res[102] = 0.0;
    res[103] = 0.0;
    res[104] = Qaux[0]*((-Q[7]) + (Q[9]/5.0));
    res[105] = t0*(t8 - 7.0*Q[8]);
    res[106] = (Qaux[0]*t10/105.0);
    res[107] = (-Q[10]*t2);
    res[108] = 0.0;
    res[109] = 0.0;
    res[110] = 0.0;
    res[111] = 0.0;
    res[112] = 0.0;
    res[113] = 0.0;
    res[114] = 0.0;
    res[115] = 0.0;
    res[116] = Qaux[0]*((-Q[8]) + (3.0/7.0)*Q[10]);
    res[117] = Qaux[0]*((-Q[7]) - (Q[9]/7.0) + (4.0/21.0)*Q[11]);
    res[118] = (-t11*t2);
    res[119] = (-(t12/231.0));
    res[120] = 0.0;
    res[121] = 0.0;
    res[122] = 0.0;
    res[123] = 0.0;
    res[124] = 0.0;
    res[125] = 0.0;
    res[126] = 0.0;
    res[127] = 0.0;
    res[128] = t10*t5;
    res[129] = (-t11*t5);
    res[130] = (-Qaux[0]*(Q[7] + (Q[9]/5.0) + (Q[11]/33.0)));
    res[131] = (-(t13/33.0));
    res[132] = 0.0;
    res[133] = 0.0;
    res[134] = 0.0;
    res[135] = 0.0;
    res[136] = 0.0;
    res[137] = 0.0;
    res[138] = 0.0;
    res[139] = 0.0;
    res[140] = (-Q[10]*t7);
    res[141] = (-(2.0/77.0)*t12);
    res[142] = (-(5.0/77.0)*t13);
    res[143] = (-Qaux[0]*(Q[7] + (17.0/77.0)*Q[9] + (81.0/1001.0)*Q[11]));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> eigenvalues(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T* n)
    {
    T t0 = std::max((T)1e-14, Q[1]);
    T t1 = (1.0/(t0));
    T t2 = std::sqrt((((Q[3]*n[0] + Q[8]*n[1])*(Q[3]*n[0] + Q[8]*n[1])) + (((Q[11]*n[1] + Q[6]*n[0])*(Q[11]*n[1] + Q[6]*n[0]))/3.0) + (3.0/5.0)*((Q[4]*n[0] + Q[9]*n[1])*(Q[4]*n[0] + Q[9]*n[1])) + (3.0/7.0)*((Q[10]*n[1] + Q[5]*n[0])*(Q[10]*n[1] + Q[5]*n[0])) + (p[0]*std::max((T)0.0, (Q[1]*Q[1]*Q[1]*Q[1]*Q[1]))/(t0*t0))));
    T t3 = (Q[2]*n[0] + Q[7]*n[1]);
    T t4 = t1*t3;
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = t1*(t3 - t2);
    res[2] = t1*(t2 + t3);
    res[3] = t4;
    res[4] = t4;
    res[5] = t4;
    res[6] = t4;
    res[7] = t4;
    res[8] = t4;
    res[9] = t4;
    res[10] = t4;
    res[11] = t4;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> source(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T dt,
        const T* X)
    {
    T t0 = (1.0/(p[2]));
    T t1 = t0*(Q[2] + Q[3] + Q[4] + Q[5] + Q[6]);
    T t2 = Qaux[0]*p[1];
    T t3 = (Qaux[0]*Qaux[0]);
    T t4 = p[0]*std::pow(Qaux[0], (4.0/3.0))*(p[3]*p[3])*std::sqrt((1e-24 + t3*(Q[2]*Q[2]) + t3*(Q[7]*Q[7])));
    T t5 = 4.0*Qaux[0];
    T t6 = (t1 + Q[3]*t5);
    T t7 = 3.0*t2;
    T t8 = 12.0*Qaux[0];
    T t9 = (t1 + Q[4]*t8);
    T t10 = 5.0*t2;
    T t11 = 24.0*Qaux[0];
    T t12 = 7.0*t2;
    T t13 = 40.0*Qaux[0];
    T t14 = 9.0*t2;
    T t15 = t0*(Q[10] + Q[11] + Q[7] + Q[8] + Q[9]);
    T t16 = (t15 + Q[8]*t5);
    T t17 = (t15 + Q[9]*t8);
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = 0.0;
    res[2] = ((-Q[2]*t4) - t1*t2 + Q[1]*p[0]*p[4]);
    res[3] = (-t7*(t6 + Q[5]*t5));
    res[4] = (-t10*(t9 + Q[6]*t8));
    res[5] = (-t12*(t6 + Q[5]*t11));
    res[6] = (-t14*(t9 + Q[6]*t13));
    res[7] = ((-Q[7]*t4) - t15*t2 + Q[1]*p[0]*p[5]);
    res[8] = (-t7*(t16 + Q[10]*t5));
    res[9] = (-t10*(t17 + Q[11]*t8));
    res[10] = (-t12*(t16 + Q[10]*t11));
    res[11] = (-t14*(t17 + Q[11]*t13));
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 24> flux(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = ((Q[3]*Q[3])/3.0);
    T t1 = (Q[4]*Q[4]);
    T t2 = (Q[5]*Q[5]);
    T t3 = (Q[6]*Q[6]);
    T t4 = Q[3]*Q[4];
    T t5 = Q[4]*Q[5];
    T t6 = Q[5]*Q[6];
    T t7 = 2.0*Qaux[0];
    T t8 = Q[3]*Q[5];
    T t9 = Q[4]*Q[6];
    T t10 = (4.0/9.0)*Q[3];
    T t11 = Q[10]*Q[5];
    T t12 = Q[11]*Q[6];
    T t13 = Q[3]*Q[8];
    T t14 = Q[4]*Q[9];
    T t15 = Qaux[0]*((t13/3.0) + (t14/5.0) + (t11/7.0) + (t12/9.0) + Q[2]*Q[7]);
    T t16 = Q[10]*Q[4];
    T t17 = Q[10]*Q[6];
    T t18 = Q[11]*Q[5];
    T t19 = Q[3]*Q[9];
    T t20 = Q[4]*Q[8];
    T t21 = Q[5]*Q[9];
    T t22 = Qaux[0]*((2.0/5.0)*t19 + (2.0/5.0)*t20 + (4.0/21.0)*t17 + (4.0/21.0)*t18 + (9.0/35.0)*t16 + (9.0/35.0)*t21 + Q[2]*Q[8] + Q[3]*Q[7]);
    T t23 = Q[10]*Q[3];
    T t24 = Q[11]*Q[4];
    T t25 = Q[5]*Q[8];
    T t26 = Q[6]*Q[9];
    T t27 = Qaux[0]*((2.0/3.0)*t13 + (2.0/7.0)*t14 + (2.0/7.0)*t24 + (2.0/7.0)*t26 + (3.0/7.0)*t23 + (3.0/7.0)*t25 + (4.0/21.0)*t11 + (100.0/693.0)*t12 + Q[2]*Q[9] + Q[4]*Q[7]);
    T t28 = (4.0/9.0)*Q[8];
    T t29 = Qaux[0]*((2.0/11.0)*t17 + (2.0/11.0)*t18 + (3.0/5.0)*t19 + (3.0/5.0)*t20 + (4.0/15.0)*t16 + (4.0/15.0)*t21 + Q[10]*Q[2] + Q[11]*t10 + Q[5]*Q[7] + Q[6]*t28);
    T t30 = Qaux[0]*((4.0/7.0)*t23 + (4.0/7.0)*t25 + (18.0/35.0)*t14 + (18.0/77.0)*t11 + (20.0/77.0)*t24 + (20.0/77.0)*t26 + (162.0/1001.0)*t12 + Q[11]*Q[2] + Q[6]*Q[7]);
    T t31 = (Q[10]*Q[10]);
    T t32 = (Q[11]*Q[11]);
    T t33 = ((Q[8]*Q[8])/3.0);
    T t34 = (Q[9]*Q[9]);
    T t35 = Q[10]*Q[11];
    T t36 = Q[10]*Q[9];
    T t37 = Q[8]*Q[9];
    T t38 = Q[10]*Q[8];
    T t39 = Q[11]*Q[9];
    SimpleArray<T, 24> res;
    res[0] = 0.0;
    res[1] = Q[2];
    res[2] = Qaux[0]*(t0 + (Q[2]*Q[2]) + (t1/5.0) + (t2/7.0) + (t3/9.0));
    res[3] = t7*((2.0/5.0)*t4 + (4.0/21.0)*t6 + (9.0/35.0)*t5 + Q[2]*Q[3]);
    res[4] = t7*(t0 + (t1/7.0) + (2.0/7.0)*t9 + (2.0/21.0)*t2 + (3.0/7.0)*t8 + (50.0/693.0)*t3 + Q[2]*Q[4]);
    res[5] = t7*((2.0/11.0)*t6 + (3.0/5.0)*t4 + (4.0/15.0)*t5 + Q[2]*Q[5] + Q[6]*t10);
    res[6] = t7*((4.0/7.0)*t8 + (9.0/35.0)*t1 + (9.0/77.0)*t2 + (20.0/77.0)*t9 + (81.0/1001.0)*t3 + Q[2]*Q[6]);
    res[7] = t15;
    res[8] = t22;
    res[9] = t27;
    res[10] = t29;
    res[11] = t30;
    res[12] = 0.0;
    res[13] = Q[7];
    res[14] = t15;
    res[15] = t22;
    res[16] = t27;
    res[17] = t29;
    res[18] = t30;
    res[19] = Qaux[0]*(t33 + (Q[7]*Q[7]) + (t34/5.0) + (t31/7.0) + (t32/9.0));
    res[20] = t7*((2.0/5.0)*t37 + (4.0/21.0)*t35 + (9.0/35.0)*t36 + Q[7]*Q[8]);
    res[21] = t7*(t33 + (t34/7.0) + (2.0/7.0)*t39 + (2.0/21.0)*t31 + (3.0/7.0)*t38 + (50.0/693.0)*t32 + Q[7]*Q[9]);
    res[22] = t7*((2.0/11.0)*t35 + (3.0/5.0)*t37 + (4.0/15.0)*t36 + Q[10]*Q[7] + Q[11]*t28);
    res[23] = t7*((4.0/7.0)*t38 + (9.0/35.0)*t34 + (9.0/77.0)*t31 + (20.0/77.0)*t39 + (81.0/1001.0)*t32 + Q[11]*Q[7]);
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 288> nonconservative_matrix(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = Q[1]*p[0];
    T t1 = Qaux[0]*((-Q[2]) + (Q[4]/5.0));
    T t2 = (Qaux[0]/35.0);
    T t3 = t2*((-7.0*Q[3]) + 3.0*Q[5]);
    T t4 = Qaux[0]*((-9.0*Q[4]) + 5.0*Q[6]);
    T t5 = (t4/105.0);
    T t6 = (Qaux[0]/21.0);
    T t7 = (-Q[5]*t6);
    T t8 = Qaux[0]*((-Q[3]) + (3.0/7.0)*Q[5]);
    T t9 = Qaux[0]*((-Q[2]) - (Q[4]/7.0) + (4.0/21.0)*Q[6]);
    T t10 = (Q[5] + 6.0*Q[3]);
    T t11 = (-t10*t6);
    T t12 = Qaux[0]*(5.0*Q[6] + 33.0*Q[4]);
    T t13 = (-(t12/231.0));
    T t14 = (2.0/15.0)*t4;
    T t15 = (2.0/15.0)*Qaux[0];
    T t16 = (-t10*t15);
    T t17 = (-Qaux[0]*(Q[2] + (Q[4]/5.0) + (Q[6]/33.0)));
    T t18 = Qaux[0]*(3.0*Q[5] + 11.0*Q[3]);
    T t19 = (-(t18/33.0));
    T t20 = (10.0/7.0)*Qaux[0];
    T t21 = (-Q[5]*t20);
    T t22 = (-(2.0/77.0)*t12);
    T t23 = (-(5.0/77.0)*t18);
    T t24 = (-Qaux[0]*(Q[2] + (17.0/77.0)*Q[4] + (81.0/1001.0)*Q[6]));
    T t25 = Qaux[0]*((-Q[7]) + (Q[9]/5.0));
    T t26 = 3.0*Q[10];
    T t27 = t2*(t26 - 7.0*Q[8]);
    T t28 = 5.0*Q[11];
    T t29 = (t28 - 9.0*Q[9]);
    T t30 = (Qaux[0]*t29/105.0);
    T t31 = (-Q[10]*t6);
    T t32 = Qaux[0]*((-Q[8]) + (3.0/7.0)*Q[10]);
    T t33 = Qaux[0]*((-Q[7]) - (Q[9]/7.0) + (4.0/21.0)*Q[11]);
    T t34 = (Q[10] + 6.0*Q[8]);
    T t35 = (-t34*t6);
    T t36 = Qaux[0]*(t28 + 33.0*Q[9]);
    T t37 = (-(t36/231.0));
    T t38 = t15*t29;
    T t39 = (-t15*t34);
    T t40 = (-Qaux[0]*(Q[7] + (Q[9]/5.0) + (Q[11]/33.0)));
    T t41 = Qaux[0]*(t26 + 11.0*Q[8]);
    T t42 = (-(t41/33.0));
    T t43 = (-Q[10]*t20);
    T t44 = (-(2.0/77.0)*t36);
    T t45 = (-(5.0/77.0)*t41);
    T t46 = (-Qaux[0]*(Q[7] + (17.0/77.0)*Q[9] + (81.0/1001.0)*Q[11]));
    SimpleArray<T, 288> res;
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
    res[23] = 0.0;
    res[24] = t0;
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
    res[35] = 0.0;
    res[36] = 0.0;
    res[37] = 0.0;
    res[38] = 0.0;
    res[39] = t1;
    res[40] = t3;
    res[41] = t5;
    res[42] = t7;
    res[43] = 0.0;
    res[44] = 0.0;
    res[45] = 0.0;
    res[46] = 0.0;
    res[47] = 0.0;
    res[48] = 0.0;
    res[49] = 0.0;
    res[50] = 0.0;
    res[51] = t8;
    res[52] = t9;
    res[53] = t11;
    res[54] = t13;
    res[55] = 0.0;
    res[56] = 0.0;
    res[57] = 0.0;
    res[58] = 0.0;
    res[59] = 0.0;
    res[60] = 0.0;
    res[61] = 0.0;
    res[62] = 0.0;
    res[63] = t14;
    res[64] = t16;
    res[65] = t17;
    res[66] = t19;
    res[67] = 0.0;
    res[68] = 0.0;
    res[69] = 0.0;
    res[70] = 0.0;
    res[71] = 0.0;
    res[72] = 0.0;
    res[73] = 0.0;
    res[74] = 0.0;
    res[75] = t21;
    res[76] = t22;
    res[77] = t23;
    res[78] = t24;
    res[79] = 0.0;
    res[80] = 0.0;
    res[81] = 0.0;
    res[82] = 0.0;
    res[83] = 0.0;
    res[84] = 0.0;
    res[85] = 0.0;
    res[86] = 0.0;
    res[87] = 0.0;
    res[88] = 0.0;
    res[89] = 0.0;
    res[90] = 0.0;
    res[91] = 0.0;
    res[92] = 0.0;
    res[93] = 0.0;
    res[94] = 0.0;
    res[95] = 0.0;
    res[96] = 0.0;
    res[97] = 0.0;
    res[98] = 0.0;
    res[99] = t25;
    res[100] = t27;
    res[101] = t30;
    res[102] = t31;
    res[103] = 0.0;
    res[104] = 0.0;
    res[105] = 0.0;
    res[106] = 0.0;
    res[107] = 0.0;
    res[108] = 0.0;
    res[109] = 0.0;
    res[110] = 0.0;
    res[111] = t32;
    res[112] = t33;
    res[113] = t35;
    res[114] = t37;
    res[115] = 0.0;
    res[116] = 0.0;
    res[117] = 0.0;
    res[118] = 0.0;
    res[119] = 0.0;
    res[120] = 0.0;
    res[121] = 0.0;
    res[122] = 0.0;
    res[123] = t38;
    res[124] = t39;
    res[125] = t40;
    res[126] = t42;
    res[127] = 0.0;
    res[128] = 0.0;
    res[129] = 0.0;
    res[130] = 0.0;
    res[131] = 0.0;
    res[132] = 0.0;
    res[133] = 0.0;
    res[134] = 0.0;
    res[135] = t43;
    res[136] = t44;
    res[137] = t45;
    res[138] = t46;
    res[139] = 0.0;
    res[140] = 0.0;
    res[141] = 0.0;
    res[142] = 0.0;
    res[143] = 0.0;
    res[144] = 0.0;
    res[145] = 0.0;
    res[146] = 0.0;
    res[147] = 0.0;
    res[148] = 0.0;
    res[149] = 0.0;
    res[150] = 0.0;
    res[151] = 0.0;
    res[152] = 0.0;
    res[153] = 0.0;
    res[154] = 0.0;
    res[155] = 0.0;
    res[156] = 0.0;
    res[157] = 0.0;
    res[158] = 0.0;
    res[159] = 0.0;
    res[160] = 0.0;
    res[161] = 0.0;
    res[162] = 0.0;
    res[163] = 0.0;
    res[164] = 0.0;
    res[165] = 0.0;
    res[166] = 0.0;
    res[167] = 0.0;
    res[168] = 0.0;
    res[169] = 0.0;
    res[170] = 0.0;
    res[171] = 0.0;
    res[172] = 0.0;
    res[173] = 0.0;
    res[174] = 0.0;
    res[175] = 0.0;
    res[176] = 0.0;
    res[177] = 0.0;
    res[178] = 0.0;
    res[179] = 0.0;
    res[180] = 0.0;
    res[181] = 0.0;
    res[182] = 0.0;
    res[183] = 0.0;
    res[184] = 0.0;
    res[185] = 0.0;
    res[186] = 0.0;
    res[187] = 0.0;
    res[188] = t1;
    res[189] = t3;
    res[190] = t5;
    res[191] = t7;
    res[192] = 0.0;
    res[193] = 0.0;
    res[194] = 0.0;
    res[195] = 0.0;
    res[196] = 0.0;
    res[197] = 0.0;
    res[198] = 0.0;
    res[199] = 0.0;
    res[200] = t8;
    res[201] = t9;
    res[202] = t11;
    res[203] = t13;
    res[204] = 0.0;
    res[205] = 0.0;
    res[206] = 0.0;
    res[207] = 0.0;
    res[208] = 0.0;
    res[209] = 0.0;
    res[210] = 0.0;
    res[211] = 0.0;
    res[212] = t14;
    res[213] = t16;
    res[214] = t17;
    res[215] = t19;
    res[216] = 0.0;
    res[217] = 0.0;
    res[218] = 0.0;
    res[219] = 0.0;
    res[220] = 0.0;
    res[221] = 0.0;
    res[222] = 0.0;
    res[223] = 0.0;
    res[224] = t21;
    res[225] = t22;
    res[226] = t23;
    res[227] = t24;
    res[228] = t0;
    res[229] = 0.0;
    res[230] = 0.0;
    res[231] = 0.0;
    res[232] = 0.0;
    res[233] = 0.0;
    res[234] = 0.0;
    res[235] = 0.0;
    res[236] = 0.0;
    res[237] = 0.0;
    res[238] = 0.0;
    res[239] = 0.0;
    res[240] = 0.0;
    res[241] = 0.0;
    res[242] = 0.0;
    res[243] = 0.0;
    res[244] = 0.0;
    res[245] = 0.0;
    res[246] = 0.0;
    res[247] = 0.0;
    res[248] = t25;
    res[249] = t27;
    res[250] = t30;
    res[251] = t31;
    res[252] = 0.0;
    res[253] = 0.0;
    res[254] = 0.0;
    res[255] = 0.0;
    res[256] = 0.0;
    res[257] = 0.0;
    res[258] = 0.0;
    res[259] = 0.0;
    res[260] = t32;
    res[261] = t33;
    res[262] = t35;
    res[263] = t37;
    res[264] = 0.0;
    res[265] = 0.0;
    res[266] = 0.0;
    res[267] = 0.0;
    res[268] = 0.0;
    res[269] = 0.0;
    res[270] = 0.0;
    res[271] = 0.0;
    res[272] = t38;
    res[273] = t39;
    res[274] = t40;
    res[275] = t42;
    res[276] = 0.0;
    res[277] = 0.0;
    res[278] = 0.0;
    res[279] = 0.0;
    res[280] = 0.0;
    res[281] = 0.0;
    res[282] = 0.0;
    res[283] = 0.0;
    res[284] = t43;
    res[285] = t44;
    res[286] = t45;
    res[287] = t46;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 144> source_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    T t0 = (1.0/(p[2]));
    T t1 = t0*(Q[2] + Q[3] + Q[4] + Q[5] + Q[6]);
    T t2 = (Qaux[0]*Qaux[0]);
    T t3 = p[1]*t2;
    T t4 = (Q[2]*Q[2]);
    T t5 = (Q[7]*Q[7]);
    T t6 = std::sqrt((1e-24 + t2*t4 + t2*t5));
    T t7 = p[0]*(p[3]*p[3]);
    T t8 = t6*t7;
    T t9 = (4.0/3.0)*t8*std::pow(Qaux[0], (7.0/3.0));
    T t10 = (t7/(t6));
    T t11 = t10*std::pow(Qaux[0], (13.0/3.0))*(t4 + t5);
    T t12 = t10*std::pow(Qaux[0], (10.0/3.0));
    T t13 = Qaux[0]*p[1];
    T t14 = t0*t13;
    T t15 = (t14 + t8*std::pow(Qaux[0], (4.0/3.0)));
    T t16 = (-t14);
    T t17 = (-Q[2]*Q[7]*t12);
    T t18 = 8.0*Qaux[0];
    T t19 = (t1 + Q[3]*t18);
    T t20 = 3.0*t3;
    T t21 = (-3.0*t14);
    T t22 = t13*(t0 + 4.0*Qaux[0]);
    T t23 = (-3.0*t22);
    T t24 = 24.0*Qaux[0];
    T t25 = (t1 + Q[4]*t24);
    T t26 = 5.0*t3;
    T t27 = (-5.0*t14);
    T t28 = t13*(t0 + 12.0*Qaux[0]);
    T t29 = (-5.0*t28);
    T t30 = 48.0*Qaux[0];
    T t31 = 7.0*t3;
    T t32 = (-7.0*t14);
    T t33 = (-7.0*t22);
    T t34 = (-7.0*t13*(t0 + t24));
    T t35 = 80.0*Qaux[0];
    T t36 = 9.0*t3;
    T t37 = (-9.0*t14);
    T t38 = (-9.0*t28);
    T t39 = (-9.0*t13*(t0 + 40.0*Qaux[0]));
    T t40 = t0*(Q[10] + Q[11] + Q[7] + Q[8] + Q[9]);
    T t41 = (t40 + Q[8]*t18);
    T t42 = (t40 + Q[9]*t24);
    SimpleArray<T, 144> res;
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
    res[23] = 0.0;
    res[24] = 0.0;
    res[25] = (Q[2]*t11 + Q[2]*t9 + p[0]*p[4] + t1*t3);
    res[26] = ((-t15) - t12*t4);
    res[27] = t16;
    res[28] = t16;
    res[29] = t16;
    res[30] = t16;
    res[31] = t17;
    res[32] = 0.0;
    res[33] = 0.0;
    res[34] = 0.0;
    res[35] = 0.0;
    res[36] = 0.0;
    res[37] = t20*(t19 + Q[5]*t18);
    res[38] = t21;
    res[39] = t23;
    res[40] = t21;
    res[41] = t23;
    res[42] = t21;
    res[43] = 0.0;
    res[44] = 0.0;
    res[45] = 0.0;
    res[46] = 0.0;
    res[47] = 0.0;
    res[48] = 0.0;
    res[49] = t26*(t25 + Q[6]*t24);
    res[50] = t27;
    res[51] = t27;
    res[52] = t29;
    res[53] = t27;
    res[54] = t29;
    res[55] = 0.0;
    res[56] = 0.0;
    res[57] = 0.0;
    res[58] = 0.0;
    res[59] = 0.0;
    res[60] = 0.0;
    res[61] = t31*(t19 + Q[5]*t30);
    res[62] = t32;
    res[63] = t33;
    res[64] = t32;
    res[65] = t34;
    res[66] = t32;
    res[67] = 0.0;
    res[68] = 0.0;
    res[69] = 0.0;
    res[70] = 0.0;
    res[71] = 0.0;
    res[72] = 0.0;
    res[73] = t36*(t25 + Q[6]*t35);
    res[74] = t37;
    res[75] = t37;
    res[76] = t38;
    res[77] = t37;
    res[78] = t39;
    res[79] = 0.0;
    res[80] = 0.0;
    res[81] = 0.0;
    res[82] = 0.0;
    res[83] = 0.0;
    res[84] = 0.0;
    res[85] = (Q[7]*t11 + Q[7]*t9 + p[0]*p[5] + t3*t40);
    res[86] = t17;
    res[87] = 0.0;
    res[88] = 0.0;
    res[89] = 0.0;
    res[90] = 0.0;
    res[91] = ((-t15) - t12*t5);
    res[92] = t16;
    res[93] = t16;
    res[94] = t16;
    res[95] = t16;
    res[96] = 0.0;
    res[97] = t20*(t41 + Q[10]*t18);
    res[98] = 0.0;
    res[99] = 0.0;
    res[100] = 0.0;
    res[101] = 0.0;
    res[102] = 0.0;
    res[103] = t21;
    res[104] = t23;
    res[105] = t21;
    res[106] = t23;
    res[107] = t21;
    res[108] = 0.0;
    res[109] = t26*(t42 + Q[11]*t24);
    res[110] = 0.0;
    res[111] = 0.0;
    res[112] = 0.0;
    res[113] = 0.0;
    res[114] = 0.0;
    res[115] = t27;
    res[116] = t27;
    res[117] = t29;
    res[118] = t27;
    res[119] = t29;
    res[120] = 0.0;
    res[121] = t31*(t41 + Q[10]*t30);
    res[122] = 0.0;
    res[123] = 0.0;
    res[124] = 0.0;
    res[125] = 0.0;
    res[126] = 0.0;
    res[127] = t32;
    res[128] = t33;
    res[129] = t32;
    res[130] = t34;
    res[131] = t32;
    res[132] = 0.0;
    res[133] = t36*(t42 + Q[11]*t35);
    res[134] = 0.0;
    res[135] = 0.0;
    res[136] = 0.0;
    res[137] = 0.0;
    res[138] = 0.0;
    res[139] = t37;
    res[140] = t37;
    res[141] = t38;
    res[142] = t37;
    res[143] = t39;
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> source_jacobian_wrt_aux_variables(
        const T* Q,
        const T* Qaux,
        const T* p)
    {
    SimpleArray<T, 12> res;
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
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> update_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T dt)
    {
    T t0 = 30.0*std::max((T)0.0, ((-1.0/100.0) + Q[1]));
    T t1 = (-t0);
    SimpleArray<T, 12> res;
    res[0] = Q[0];
    res[1] = Q[1];
    res[2] = std::max(t1, std::min(Q[2], t0));
    res[3] = std::max(t1, std::min(Q[3], t0));
    res[4] = std::max(t1, std::min(Q[4], t0));
    res[5] = std::max(t1, std::min(Q[5], t0));
    res[6] = std::max(t1, std::min(Q[6], t0));
    res[7] = std::max(t1, std::min(Q[7], t0));
    res[8] = std::max(t1, std::min(Q[8], t0));
    res[9] = std::max(t1, std::min(Q[9], t0));
    res[10] = std::max(t1, std::min(Q[10], t0));
    res[11] = std::max(t1, std::min(Q[11], t0));
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

    PORTABLE_FN static inline SimpleArray<T, 12> update_aux_variables_jacobian_wrt_variables(
        const T* Q,
        const T* Qaux,
        const T* p,
        const T time,
        const T* X)
    {
    T t0 = std::max((T)1e-08, Q[1]);
    T t1 = ((Q[1]*Q[1]*Q[1]*Q[1]) + (t0*t0*t0*t0));
    SimpleArray<T, 12> res;
    res[0] = 0.0;
    res[1] = (std::sqrt(2.0)*((-(2.0*((Q[1]*Q[1]*Q[1]) + (t0*t0*t0)*Heaviside(((-1e-08) + Q[1]), (1.0/2.0)))*std::max((T)0.0, Q[1])/(t1))) + Heaviside(Q[1], (1.0/2.0)))/std::sqrt(t1));
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
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> initial_condition(
        const T* X,
        const T* p)
    {
    SimpleArray<T, 12> res;
    res[0] = 1.0;
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
    return res;
    }

    PORTABLE_FN static inline SimpleArray<T, 12> boundary_conditions(
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
        T t0 = (Q[2]*n[0] + Q[7]*n[1]);
        T t1 = 2.0*n[0];
        T t2 = (Q[3]*n[0] + Q[8]*n[1]);
        T t3 = (Q[4]*n[0] + Q[9]*n[1]);
        T t4 = (Q[10]*n[1] + Q[5]*n[0]);
        T t5 = (Q[11]*n[1] + Q[6]*n[0]);
        T t6 = 2.0*n[1];
        SimpleArray<T, 12> res;
        res[0] = Q[0];
        res[1] = Q[1];
        res[2] = (Q[2] - t0*t1);
        res[3] = (Q[3] - t1*t2);
        res[4] = (Q[4] - t1*t3);
        res[5] = (Q[5] - t1*t4);
        res[6] = (Q[6] - t1*t5);
        res[7] = (Q[7] - t0*t6);
        res[8] = (Q[8] - t2*t6);
        res[9] = (Q[9] - t3*t6);
        res[10] = (Q[10] - t4*t6);
        res[11] = (Q[11] - t5*t6);
        return res;
    }
    SimpleArray<T, 12> default_res = {0};
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
