// Kernels of the IMEX strategy's step (SolverStrategies.hpp:62-128): the
// additive Runge-Kutta scheme 2E (imex_tableau.h) with the transport explicit
// (its right-hand sides G_j come from the ordinary prep / face / gather
// kernels in MODE_RHS) and the source implicit, solved per cell.  The
// operations are those of the CPU restatement in the same order, so the two
// agree bit for bit.
#pragma once
#include "imex_tableau.h"

namespace zsme {

// The implicit source at state y: y clamped and its aux updated from aux_init
// (UpdateState), the plugin's source there, zero in cells with depth below
// 1e-6 (ModularSolver::AddImplicitSourceToResidual, ModularSolver.hpp:82-124).
template <class M>
__device__ __forceinline__ void imex_source_cell(const double* y, const double* aux_init, const double* p,
                                                 double* S) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const double X0[3] = {0.0, 0.0, 0.0};
    double ys[NQ], a[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) ys[i] = y[i];
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux_init[i];
    constrain<M>(ys, a, p);
    if (NQ > 1 && ys[1] < ark2e::dry_residual) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) S[i] = 0.0;
        return;
    }
    const auto r = M::source(ys, a, p, 0.0, 0.0, X0);
#pragma unroll
    for (int i = 0; i < NQ; ++i) S[i] = r[i];
}

// y - z - hg S(y) = 0 by Newton from y = z: the Jacobian I - hg (dS/dQ + dS/dAux
// dAux/dQ) at the clamped state, the identity in cells drier than 1e-4
// (ModularSolver::FormSourceJacobian, ModularSolver.hpp:403-460); the source
// step's elimination and stopping rule.  Returns 1 when the update limit was hit.
template <class M>
__device__ int imex_solve_cell(double hg, const double* z, double* y, const double* aux_init, const double* p) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const double X0[3] = {0.0, 0.0, 0.0};
    double S[NQ], res[NQ], J[NQ * NQ], xv[NQ];
    for (int i = 0; i < NQ; ++i) y[i] = z[i];
    int iter = 0;
    for (; iter < 15; ++iter) {
        imex_source_cell<M>(y, aux_init, p, S);
        double rn = 0.0;
        for (int i = 0; i < NQ; ++i) {
            res[i] = y[i] - z[i] - hg * S[i];
            rn += res[i] * res[i];
        }
        if (sqrt(rn) < 1e-8) break;
        double ys[NQ], a[NA];
        for (int i = 0; i < NQ; ++i) ys[i] = y[i];
        for (int i = 0; i < NA; ++i) a[i] = aux_init[i];
        constrain<M>(ys, a, p);
        for (int i = 0; i < NQ * NQ; ++i) J[i] = 0.0;
        for (int i = 0; i < NQ; ++i) J[i * NQ + i] = 1.0;
        if (!(NQ > 1 && ys[1] < ark2e::dry_jacobian)) {
            const auto dSdQ = M::source_jacobian_wrt_variables(ys, a, p);
            const auto dSdA = M::source_jacobian_wrt_aux_variables(ys, a, p);
            double dAdQ[NA * NQ];
            if constexpr (HasAuxJacobian<M>::value) {
                const auto r = M::update_aux_variables_jacobian_wrt_variables(ys, a, p);
                for (int e = 0; e < NA * NQ; ++e) dAdQ[e] = r[e];
            } else {   // forward differences, SourceStep.hpp:16-53
                const auto a0 = M::update_aux_variables(ys, a, p, 0.0, X0);
                for (int j = 0; j < NQ; ++j) {
                    double qp[NQ];
                    for (int mm = 0; mm < NQ; ++mm) qp[mm] = ys[mm];
                    const double hh = 1e-7 * (fabs(ys[j]) + 1e-7);
                    qp[j] += hh;
                    const auto a1 = M::update_aux_variables(qp, a, p, 0.0, X0);
                    for (int k = 0; k < NA; ++k) dAdQ[k * NQ + j] = (a1[k] - a0[k]) / hh;
                }
            }
            for (int i = 0; i < NQ; ++i)
                for (int j = 0; j < NQ; ++j) {
                    double term = dSdQ[i * NQ + j];
                    for (int k = 0; k < NA; ++k) term += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                    J[i * NQ + j] -= hg * term;
                }
        }
        for (int i = 0; i < NQ; ++i) res[i] = -res[i];
        if (!gepp_full<NQ>(J, res, xv)) break;
        for (int i = 0; i < NQ; ++i) y[i] += xv[i];
    }
    return iter >= 15 ? 1 : 0;
}

// The right-hand sides and implicit derivatives of the stages before stage i.
struct ImexTerms {
    const double* G[3];
    const double* S[3];
    double a[3], at[3];
    int n;
};

// out = x + h (sum_j a_j G_j + sum_j at_j S_j) for cell c, component i
__device__ __forceinline__ double imex_combination(const ImexTerms& tm, const double* x, double h, size_t id) {
    double acc = 0.0;
    for (int j = 0; j < tm.n; ++j) acc += tm.a[j] * tm.G[j][id];
    for (int j = 0; j < tm.n; ++j) acc += tm.at[j] * tm.S[j][id];
    return x[id] + h * acc;
}

// S_out = the implicit source of state x (the explicit first stage)
template <class M>
__global__ void __launch_bounds__(128) imex_source_kernel(MeshDev m, const double* __restrict__ x,
                                                          const double* __restrict__ aux,
                                                          const double* __restrict__ params,
                                                          double* __restrict__ S_out, const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    double y[NQ], a[NA], S[NQ];
    load_q<NQ>(x, C, c, y);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    imex_source_cell<M>(y, a, params + (size_t)I * m.np, S);
#pragma unroll
    for (int i = 0; i < NQ; ++i) S_out[(size_t)i * C + c] = S[i];
}

// An implicit stage: Z = x + h (sum a_j G_j + sum at_j S_j), Y solving
// Y - h gamma S(Y) = Z, its implicit derivative (Y - Z) / (h gamma) (the value
// PETSc's ARKIMEX carries to later stages).  Newton iteration limits are
// counted in diag[2].
template <class M>
__global__ void __launch_bounds__(64) imex_stage_kernel(MeshDev m, ImexTerms tm, const double* __restrict__ x,
                                                        const double* __restrict__ aux,
                                                        const double* __restrict__ params,
                                                        const double* __restrict__ dt_step,
                                                        const int* __restrict__ active, double* __restrict__ Y_out,
                                                        double* __restrict__ S_out, int* diag) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double h = dt_step[I];
    const double hg = h * ark2e::gamma;
    double z[NQ], y[NQ], a[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) z[i] = imex_combination(tm, x, h, (size_t)i * C + c);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    if (imex_solve_cell<M>(hg, z, y, a, params + (size_t)I * m.np)) atomicAdd(&diag[2], 1);
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const size_t id = (size_t)i * C + c;
        Y_out[id] = y[i];
        S_out[id] = (y[i] - z[i]) / hg;
    }
}

// The step's update x <- x + h sum_j b_j (G_j + S_j) (tm carries b in a and at)
template <class M>
__global__ void __launch_bounds__(128) imex_final_kernel(MeshDev m, ImexTerms tm, double* __restrict__ x,
                                                         const double* __restrict__ dt_step,
                                                         const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double h = dt_step[I];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const size_t id = (size_t)i * C + c;
        x[id] = imex_combination(tm, x, h, id);
    }
}

}  // namespace zsme
