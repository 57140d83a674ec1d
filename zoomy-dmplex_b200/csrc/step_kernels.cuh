// Device kernels of the SME step, templated on a generated model plugin
// (Model<T>, Numerics<T>).  All state lives in HBM as one FP64 array per
// variable ("SoA"), cells in Hilbert order.
//
// One SSP stage = prep_kernel + flux_kernel:
//   prep_kernel  per cell: wet/dry clamp of the stage state, neighbour bounds
//                of the clamped state, gradient of the unclamped state
//                (least squares or Green-Gauss), limited linear
//                reconstruction at each of the cell's faces -> face states
//                (TransportStep.hpp:196-230, 122-154, 339; Gradient.hpp;
//                Reconstruction.hpp:203-243)
//   flux_kernel  per cell: Riemann flux + fluctuations of each face from the
//                two face states, accumulated in the reference's face order
//                (TransportStep.hpp:383-565), / volume, fused with the
//                SSP-RK(s,2) stage combination
// After the last stage:
//   finalize_kernel per cell: constraints, implicit Newton source, constraints
//                (MUSCLSolver.hpp:153-186, SourceStep.hpp:125-242), CFL ratio
//                r_c / lambda_c and a per-block minimum (VirtualSolver.hpp:285-357)
//   end_step_kernel: global minimum -> next dt, time advance, dt of the next
//                step clamped to t_end (MUSCLSolver.hpp:141-149)
#pragma once
#include <cfloat>
#include <cstdint>

namespace zsme {

// ------------------------------------------------------------------ layout
struct MeshDev {
    int C;                 // cells
    int K;                 // face slots per cell
    const int* slot_nbr;   // [K][C] neighbour cell, -1 boundary, -2 no face
    const int* slot_meta;  // [K][C] bits 0-1 neighbour's slot, bit 2 "cell is support[0]",
                           //        bits 3..: bc index + 2 (0 = no condition, 1 = interior)
    const int* slot_face;  // [K][C] face id (new numbering)
    const double* slot_dx; // [K][2][C] face centroid - cell centroid
    const double* slot_w;  // [K][2][C] least-squares weights (0 where no neighbour)
    const double* vol;     // [C]
    const double* rc;      // [C] min |x_c - x_f| over the cell's faces
    const int* order;      // [C] slot permutation by increasing original face id (2 bits/slot)
    const double* fn;      // [2][F] unit normal
    const double* farea;   // [F]
    const double* fc;      // [2][F] face centroid
    const double* fnr;     // [2][F] area-weighted normal as given (Green-Gauss)
    int F;
};

struct StepDev {
    double* t;             // simulated time
    double* dt_cfl;        // CFL dt of the current state
    double* dt_step;       // dt of the step being taken (clamped to t_end), 0 if inactive
    int* active;           // 1 while t < t_end
    const double* dts;     // imposed dts (or nullptr)
    int* step_idx;         // steps taken (index into dts)
    double t_end, cfl, dt_max;
    double* partial;       // per-block CFL minima
    int n_partial;
    int* diag;             // [0] nonfinite, [1] negative depth, [2] newton unconverged
};

enum StageMode { MODE_RHS = 0, MODE_FIRST = 1, MODE_MID = 2, MODE_FINAL = 3, MODE_EULER = 4 };

struct Opts {
    int order;     // reconstruction order
    int limiter;   // 0 none, 1 vacuum + tvd
    int gradient;  // 0 green-gauss, 1 least squares
    int stages;    // s of SSP-RK(s,2)
    int source;    // operator-split source
};

__device__ __forceinline__ int meta_nslot(int m) { return m & 3; }
__device__ __forceinline__ bool meta_isL(int m) { return (m >> 2) & 1; }
__device__ __forceinline__ int meta_bc(int m) { return (m >> 3) - 2; }

// ---------------------------------------------------------- cell helpers
template <class M>
__device__ __forceinline__ void constrain(double* q, double* a, const double* p) {
    if constexpr (HasUpdateVariables<M>::value) {
        auto r = M::update_variables(q, a, p, 0.0);
#pragma unroll
        for (int i = 0; i < M::n_dof_q; ++i) q[i] = r[i];
    }
    const double X0[3] = {0.0, 0.0, 0.0};
    auto ra = M::update_aux_variables(q, a, p, 0.0, X0);
#pragma unroll
    for (int i = 0; i < M::n_dof_qaux; ++i) a[i] = ra[i];
}

template <int NQ>
__device__ __forceinline__ void load_q(const double* __restrict__ w, int C, int c, double* q) {
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = w[(size_t)i * C + c];
}

// LinearReconstructor::Reconstruct with VacuumLimiter + TVDLimiter
// (Reconstruction.hpp:25-36, 62-81, 203-243): one scalar alpha per face.
template <int NQ, int DIM>
__device__ __forceinline__ void reconstruct(const double* q, const double* g, const double* dx,
                                            const double* qmin, const double* qmax, int limiter,
                                            double* out) {
    double delta[NQ];
    double alpha = 1.0;
    bool vac = limiter && NQ > 1 && qmin[1] < 1e-2;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        double d = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) d += g[i * DIM + k] * dx[k];
        delta[i] = d;
        if (limiter) {
            double qfu = q[i] + d;
            double dq = qfu - q[i];
            double al = 1.0;
            if (!(fabs(dq) < 1e-12)) {
                if (dq > 0) al = (qmax[i] > q[i]) ? fmin(1.0, (qmax[i] - q[i]) / dq) : 0.0;
                else al = (qmin[i] < q[i]) ? fmin(1.0, (qmin[i] - q[i]) / dq) : 0.0;
            }
            // alpha = min over components of min(vacuum, tvd) (NaN-ignoring as "<")
            if (al < alpha) alpha = al;
        }
    }
    if (vac) alpha = 0.0 < alpha ? 0.0 : alpha;
#pragma unroll
    for (int i = 0; i < NQ; ++i) out[i] = q[i] + alpha * delta[i];
}

// ----------------------------------------------------------------- prep
template <class M>
__global__ void __launch_bounds__(128) prep_kernel(MeshDev m, Opts o, const double* __restrict__ w,
                                                   const double* __restrict__ aux, const double* __restrict__ p,
                                                   double* __restrict__ fs, const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, DIM = M::dimension;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || (active && !*active)) return;
    double qg[NQ], ql[NQ], a[NA];
    load_q<NQ>(w, C, c, qg);
#pragma unroll
    for (int i = 0; i < NQ; ++i) ql[i] = qg[i];
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    constrain<M>(ql, a, p);
    if (o.order < 2) {
        for (int k = 0; k < m.K; ++k) {
            if (m.slot_face[k * C + c] < 0) continue;
#pragma unroll
            for (int i = 0; i < NQ; ++i) fs[((size_t)k * NQ + i) * C + c] = ql[i];
        }
        return;
    }
    double mn[NQ], mx[NQ], g[NQ * DIM];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        mn[i] = ql[i];
        mx[i] = ql[i];
    }
#pragma unroll
    for (int i = 0; i < NQ * DIM; ++i) g[i] = 0.0;
    // neighbours in cone order: bounds of the clamped state, LSQ of the raw state
    for (int k = 0; k < m.K; ++k) {
        const int n = m.slot_nbr[k * C + c];
        if (n < 0) continue;
        double qn[NQ], an[NA];
        load_q<NQ>(w, C, n, qn);
        double wk[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[((size_t)k * 2 + d) * C + c];
        if (o.gradient == 1) {
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                double du = qn[i] - qg[i];
#pragma unroll
                for (int d = 0; d < DIM; ++d) g[i * DIM + d] += wk[d] * du;
            }
        }
#pragma unroll
        for (int i = 0; i < NA; ++i) an[i] = aux[(size_t)i * C + n];
        constrain<M>(qn, an, p);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            if (qn[i] < mn[i]) mn[i] = qn[i];
            if (qn[i] > mx[i]) mx[i] = qn[i];
        }
    }
    if (o.gradient == 0) {
        // Green-Gauss in increasing original face order (Gradient.hpp:91-176)
        const int ord = m.order[c];
        for (int j = 0; j < m.K; ++j) {
            const int k = (ord >> (2 * j)) & 3;
            const int f = m.slot_face[k * C + c];
            if (f < 0) continue;
            const int meta = m.slot_meta[k * C + c];
            const int n = m.slot_nbr[k * C + c];
            const double Nf[2] = {m.fnr[f], m.fnr[m.F + f]};
            if (n >= 0) {
                double qn[NQ];
                load_q<NQ>(w, C, n, qn);
                const bool isL = meta_isL(meta);
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    double fv = 0.5 * (isL ? (qg[i] + qn[i]) : (qn[i] + qg[i]));
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        double v = fv * Nf[d];
                        if (isL) g[i * DIM + d] += v;
                        else g[i * DIM + d] -= v;
                    }
                }
            } else if (meta_bc(meta) >= 0) {
                double nh[3] = {m.fn[f], m.fn[m.F + f], 0.0};
                double xf[3] = {m.fc[f], m.fc[m.F + f], 0.0};
                auto qb = M::boundary_conditions(meta_bc(meta), qg, (const double*)nullptr, p, nh, xf, 0.0, 0.0);
#pragma unroll
                for (int i = 0; i < NQ; ++i)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[i * DIM + d] += qb[i] * Nf[d];
            }
        }
        const double v = m.vol[c];
        if (v > 1e-15) {
#pragma unroll
            for (int i = 0; i < NQ * DIM; ++i) g[i] /= v;
        }
    }
    for (int k = 0; k < m.K; ++k) {
        if (m.slot_face[k * C + c] < 0) continue;
        double dx[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) dx[d] = m.slot_dx[((size_t)k * 2 + d) * C + c];
        double qf[NQ];
        reconstruct<NQ, DIM>(ql, g, dx, mn, mx, o.limiter, qf);
#pragma unroll
        for (int i = 0; i < NQ; ++i) fs[((size_t)k * NQ + i) * C + c] = qf[i];
    }
}

// ----------------------------------------------------------------- flux
template <class M, class N>
__global__ void __launch_bounds__(128) flux_kernel(MeshDev m, Opts o, const double* __restrict__ fs,
                                                   const double* __restrict__ aux, const double* __restrict__ p,
                                                   int mode, double t_host, const double* t_dev,
                                                   double stage_frac, const double* x_in, double* x_out,
                                                   double* base, const double* __restrict__ dt_step,
                                                   const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || (active && !*active)) return;
    double acc[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
    double ac[NA];
#pragma unroll
    for (int i = 0; i < NA; ++i) ac[i] = aux[(size_t)i * C + c];
    // stage time t0 + dt * i/(s-1) (TSSSPStep_RK_2); only time-dependent
    // boundary conditions / aux see it
    const double t = t_dev ? (*t_dev + stage_frac * (dt_step ? *dt_step : 0.0)) : t_host;
    const int ord = m.order[c];
    for (int j = 0; j < m.K; ++j) {
        const int k = (ord >> (2 * j)) & 3;
        const int f = m.slot_face[k * C + c];
        if (f < 0) continue;
        const int meta = m.slot_meta[k * C + c];
        const int n = m.slot_nbr[k * C + c];
        const int bc = meta_bc(meta);
        if (n < 0 && bc < 0) continue;  // exterior face without a condition: no flux
        const double area = m.farea[f];
        const double nh[3] = {m.fn[f], m.fn[m.F + f], 0.0};
        const double xf[3] = {m.fc[f], m.fc[m.F + f], 0.0};
        double qo[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qo[i] = fs[((size_t)k * NQ + i) * C + c];
        if (n >= 0) {
            const int ks = meta_nslot(meta);
            double qn[NQ], an[NA];
#pragma unroll
            for (int i = 0; i < NQ; ++i) qn[i] = fs[((size_t)ks * NQ + i) * C + n];
#pragma unroll
            for (int i = 0; i < NA; ++i) an[i] = aux[(size_t)i * C + n];
            const bool isL = meta_isL(meta);
            const double* qL = isL ? qo : qn;
            const double* qR = isL ? qn : qo;
            double aL[NA], aR[NA];
            {
                auto ra = M::update_aux_variables(qL, isL ? ac : an, p, 0.0, xf);
                auto rb = M::update_aux_variables(qR, isL ? an : ac, p, 0.0, xf);
#pragma unroll
                for (int i = 0; i < NA; ++i) { aL[i] = ra[i]; aR[i] = rb[i]; }
            }
            auto flux = N::numerical_flux(qL, qR, aL, aR, p, nh);
            auto nc = N::numerical_fluctuations(qL, qR, aL, aR, p, nh);
            if (isL) {
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= nc[NQ + i] * area;
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= flux[i] * area;
            } else {
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= nc[i] * area;
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] += flux[i] * area;
            }
        } else {
            double aL[NA], aR[NA];
            auto ra = M::update_aux_variables(qo, ac, p, t, xf);
#pragma unroll
            for (int i = 0; i < NA; ++i) aL[i] = ra[i];
            auto qR = M::boundary_conditions(bc, qo, aL, p, nh, xf, t, 0.0);
            auto rb = M::update_aux_variables(qR.data, aL, p, t, xf);
#pragma unroll
            for (int i = 0; i < NA; ++i) aR[i] = rb[i];
            auto flux = N::numerical_flux(qo, qR.data, aL, aR, p, nh);
            auto nc = N::numerical_fluctuations(qo, qR.data, aL, aR, p, nh);
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= nc[NQ + i] * area;
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= flux[i] * area;
        }
    }
    const double v = m.vol[c];
    if (v > 1e-15) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) acc[i] /= v;
    }
    // SSP-RK(s,2) stage combination (PETSc TSSSPStep_RK_2) / forward Euler
    const double h = dt_step ? *dt_step : 0.0;
    const int s = o.stages;
    switch (mode) {
        case MODE_RHS:
#pragma unroll
            for (int i = 0; i < NQ; ++i) x_out[(size_t)i * C + c] = acc[i];
            break;
        case MODE_FIRST: {  // w = x + dt/(s-1) F
            const double a = h / (s - 1.);
#pragma unroll
            for (int i = 0; i < NQ; ++i) x_out[(size_t)i * C + c] = x_in[(size_t)i * C + c] + a * acc[i];
            break;
        }
        case MODE_MID: {    // w += dt/(s-1) F (in place)
            const double a = h / (s - 1.);
#pragma unroll
            for (int i = 0; i < NQ; ++i) x_out[(size_t)i * C + c] = x_in[(size_t)i * C + c] + a * acc[i];
            break;
        }
        case MODE_FINAL: {  // X = (s-1)/s w + dt/s F + 1/s X
            const double al = (s - 1.) / s, be = h / s, ga = 1. / s;
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const size_t id = (size_t)i * C + c;
                base[id] = al * x_in[id] + be * acc[i] + ga * base[id];
            }
            break;
        }
        case MODE_EULER: {  // X = X + dt F
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const size_t id = (size_t)i * C + c;
                base[id] = base[id] + h * acc[i];
            }
            break;
        }
    }
}

// ---------------------------------------------------------------- source
// SourceStep::SolveLocalCell (SourceStep.hpp:125-209) with the GEPP of
// SolveLinearSystem (211-242); dAux/dQ as aux_jacobian_wrt_q (26-53).
template <class M>
__device__ __forceinline__ int newton_cell(double dtl, double* q, double* aux, const double* p) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const double X0[3] = {0.0, 0.0, 0.0};
    double q_old[NQ], res[NQ], J[NQ * NQ], delta[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q_old[i] = q[i];
    int iter = 0;
    for (; iter < 15; ++iter) {
        {
            auto ua = M::update_aux_variables(q, aux, p, 0.0, X0);
#pragma unroll
            for (int i = 0; i < NA; ++i) aux[i] = ua[i];
        }
        double rn = 0.0;
        {
            auto S = M::source(q, aux, p, 0.0, dtl, X0);
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                res[i] = q[i] - q_old[i] - dtl * S[i];
                rn += res[i] * res[i];
            }
        }
        if (sqrt(rn) < 1e-8) break;
        {
            auto dSdQ = M::source_jacobian_wrt_variables(q, aux, p);
            auto dSdA = M::source_jacobian_wrt_aux_variables(q, aux, p);
            double dAdQ[NA * NQ];
            if constexpr (HasAuxJacobian<M>::value) {
                auto r = M::update_aux_variables_jacobian_wrt_variables(q, aux, p);
#pragma unroll
                for (int i = 0; i < NA * NQ; ++i) dAdQ[i] = r[i];
            } else {
                auto a0 = M::update_aux_variables(q, aux, p, 0.0, X0);
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    double qp[NQ];
#pragma unroll
                    for (int mm = 0; mm < NQ; ++mm) qp[mm] = q[mm];
                    const double hh = 1e-7 * (fabs(q[j]) + 1e-7);
                    qp[j] += hh;
                    auto a1 = M::update_aux_variables(qp, aux, p, 0.0, X0);
#pragma unroll
                    for (int k = 0; k < NA; ++k) dAdQ[k * NQ + j] = (a1[k] - a0[k]) / hh;
                }
            }
#pragma unroll
            for (int i = 0; i < NQ; ++i)
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    double term = dSdQ[i * NQ + j];
#pragma unroll
                    for (int k = 0; k < NA; ++k) term += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                    J[i * NQ + j] = (i == j ? 1.0 : 0.0) - dtl * term;
                }
        }
#pragma unroll
        for (int i = 0; i < NQ; ++i) res[i] = -res[i];
        // Gaussian elimination with partial pivoting
        bool ok = true;
        for (int k = 0; k < NQ && ok; ++k) {
            int mr = k;
            double mv = fabs(J[k * NQ + k]);
            for (int i = k + 1; i < NQ; ++i)
                if (fabs(J[i * NQ + k]) > mv) { mv = fabs(J[i * NQ + k]); mr = i; }
            if (mv < 1e-14) { ok = false; break; }
            if (mr != k) {
                for (int j = k; j < NQ; ++j) { double tt = J[k * NQ + j]; J[k * NQ + j] = J[mr * NQ + j]; J[mr * NQ + j] = tt; }
                double tt = res[k]; res[k] = res[mr]; res[mr] = tt;
            }
            for (int i = k + 1; i < NQ; ++i) {
                const double fct = J[i * NQ + k] / J[k * NQ + k];
                for (int j = k; j < NQ; ++j) J[i * NQ + j] -= fct * J[k * NQ + j];
                res[i] -= fct * res[k];
            }
        }
        if (!ok) break;
        for (int i = NQ - 1; i >= 0; --i) {
            double sum = 0.0;
            for (int j = i + 1; j < NQ; ++j) sum += J[i * NQ + j] * delta[j];
            delta[i] = (res[i] - sum) / J[i * NQ + i];
        }
#pragma unroll
        for (int i = 0; i < NQ; ++i) q[i] += delta[i];
    }
    return iter >= 15 ? 1 : 0;
}

// ------------------------------------------------------------- finalize
enum FinalizeFlags {
    FIN_PRE = 1,     // constraints after the transport update (MUSCLSolver.hpp:153)
    FIN_SOURCE = 2,  // implicit source over dt_src (SourceStep::Solve), then constraints if FIN_PRE
    FIN_POST = 4,    // constraints of PostStep (VirtualSolver.hpp:128-150)
    FIN_DT = 8,      // CFL ratio + per-block minimum
    FIN_WRITE = 16,  // store the state / aux back
};

template <class M, class N>
__global__ void __launch_bounds__(128) finalize_kernel(MeshDev m, double* __restrict__ x, double* __restrict__ aux,
                                                       const double* __restrict__ p, StepDev sd,
                                                       const double* __restrict__ dt_src, int flags) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, DIM = M::dimension;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double ratio = DBL_MAX;
    const bool act = sd.active ? (*sd.active != 0) : true;
    if (c < C && act) {
        double q[NQ], a[NA];
        load_q<NQ>(x, C, c, q);
#pragma unroll
        for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
        if (flags & FIN_PRE) constrain<M>(q, a, p);
        if (flags & FIN_SOURCE) {
            if (newton_cell<M>(*dt_src, q, a, p)) atomicAdd(&sd.diag[2], 1);
            if (flags & FIN_PRE) constrain<M>(q, a, p);
        }
        if (flags & FIN_POST) constrain<M>(q, a, p);
        if (flags & FIN_WRITE) {
#pragma unroll
            for (int i = 0; i < NQ; ++i) x[(size_t)i * C + c] = q[i];
#pragma unroll
            for (int i = 0; i < NA; ++i) aux[(size_t)i * C + c] = a[i];
            bool bad = false;
#pragma unroll
            for (int i = 0; i < NQ; ++i) bad |= !isfinite(q[i]);
            if (bad) atomicAdd(&sd.diag[0], 1);
            if (q[1] < -1e-10) atomicAdd(&sd.diag[1], 1);
        }
        if (flags & FIN_DT) {
            double eig = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double n[3] = {0.0, 0.0, 0.0};
                n[d] = 1.0;
                auto r = N::local_max_abs_eigenvalue(q, a, p, n);
                if (r[0] > eig) eig = r[0];
            }
            if (!(eig < 1e-14)) {
                const double rcv = m.rc[c];
                if (rcv < DBL_MAX) ratio = rcv / eig;
            }
        }
    }
    if (!(flags & FIN_DT)) return;
    // block minimum (a NaN ratio never wins a "<" comparison, as in the reference)
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) {
        double o2 = __shfl_down_sync(0xffffffffu, ratio, off);
        if (o2 < ratio) ratio = o2;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ratio;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        double r = threadIdx.x < nw ? red[threadIdx.x] : DBL_MAX;
        for (int off = 16; off > 0; off >>= 1) {
            double o2 = __shfl_down_sync(0xffffffffu, r, off);
            if (o2 < r) r = o2;
        }
        if (threadIdx.x == 0) sd.partial[blockIdx.x] = r;
    }
}

// --------------------------------------------------------------- step ends
// begin: dt of this step from the CFL dt (or the imposed one), clamped to
// land on t_end; inactive once t >= t_end.
static __global__ void begin_step_kernel(StepDev sd) {
    const double t0 = *sd.t;
    double d0 = sd.dts ? sd.dts[*sd.step_idx] : *sd.dt_cfl;
    const int act = t0 < sd.t_end;
    if (t0 + d0 > sd.t_end) d0 = sd.t_end - t0;
    *sd.active = act;
    *sd.dt_step = act ? d0 : 0.0;
}

// end: global min of the per-block ratios -> CFL dt; time advance.
static __global__ void end_step_kernel(StepDev sd, int advance, double min_dt_floor) {
    double r = DBL_MAX;
    for (int i = threadIdx.x; i < sd.n_partial; i += blockDim.x) {
        const double v = sd.partial[i];
        if (v < r) r = v;
    }
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) {
        double o2 = __shfl_down_sync(0xffffffffu, r, off);
        if (o2 < r) r = o2;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            if (red[w] < r) r = red[w];
        double dt;
        if (!isfinite(r) || r >= 0.5 * DBL_MAX) dt = sd.dt_max;
        else dt = sd.cfl * r;
        if (advance) {
            if (*sd.active) {
                *sd.t = *sd.t + *sd.dt_step;
                *sd.step_idx += 1;
                *sd.dt_cfl = dt;
            }
        } else {
            *sd.dt_cfl = dt > min_dt_floor ? dt : min_dt_floor;
        }
    }
}

// ------------------------------------------------------- layout transforms
// AoS (caller order) <-> SoA (Hilbert order)
static __global__ void aos_to_soa_kernel(const double* __restrict__ aos, double* __restrict__ soa, const int* __restrict__ old_of_new,
                                  int C, int nq) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int o = old_of_new[c];
    for (int i = 0; i < nq; ++i) soa[(size_t)i * C + c] = aos[(size_t)o * nq + i];
}
static __global__ void soa_to_aos_kernel(const double* __restrict__ soa, double* __restrict__ aos, const int* __restrict__ old_of_new,
                                  int C, int nq) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int o = old_of_new[c];
    for (int i = 0; i < nq; ++i) aos[(size_t)o * nq + i] = soa[(size_t)i * C + c];
}

}  // namespace zsme
