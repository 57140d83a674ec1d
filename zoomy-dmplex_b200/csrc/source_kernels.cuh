// Constraints, implicit per-cell source and the CFL ratio of one time step.
//
// The Newton iteration is SourceStep::SolveLocalCell (SourceStep.hpp:125-209)
// with the Gaussian elimination with partial pivoting (GEPP) of
// SolveLinearSystem (211-242), operation for operation.
//
// Register fast path.  For SME-layout models (Q = [b, h, moments of
// direction 1, moments of direction 2]) the Newton matrix
// J = I - dt (dS/dQ + dS/dAux dAux/dQ) usually has this structure:
//   (a) dS/dAux is zero in every entry and the state is finite, so the
//       chain-rule term vanishes and dAux/dQ need not be formed;
//   (b) the b and h rows of dS/dQ and of the residual are zero (rows 0 and 1
//       of J are unit rows, right-hand side zero there), and dS/dQ has no
//       b column;
//   (c) |J[i][1]| <= 1 for the momentum rows, so GEPP never swaps a momentum
//       row into pivot position 1;
//   (d) optionally, the two directions' moment blocks do not couple.
// Under (a)-(c) GEPP's first two eliminations change nothing but the signs
// of zero entries, and under (d) its pivot searches and row updates never
// mix the direction blocks; the full GEPP then equals GEPP on each block
// alone, with the same operations in the same order.  Those blocks are
// small (L+1 moments per direction) and are solved fully unrolled in
// registers.  When any condition fails the generic full-size GEPP runs.
#pragma once

#include "gepp_regs.h"

namespace zsme {

template <class M>
struct SmeLayout {
    static constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    static constexpr bool ok = M::idx_b == 0 && M::idx_h == 1 && NQ > 2 && (NQ - 2) % DIM == 0;
    static constexpr int NM = ok ? (NQ - 2) / DIM : 1;   // moments per direction
    static constexpr int NB = NQ - 2;                      // momentum block
};

// One Newton update on the fast path; returns 1 if q was updated, 0 to fall
// back to the generic path (structure not met, or a singular / non-finite
// pivot, which the generic path then handles exactly as the reference).
template <class M>
__device__ __forceinline__ int newton_fast(double dtl, double* q, const double* res,
                                           const SimpleArray<double, M::n_dof_q * M::n_dof_q>& S) {
    using L = SmeLayout<M>;
    constexpr int NQ = L::NQ, NM = L::NM, NB = L::NB, DIM = L::DIM;
    if constexpr (!L::ok) {
        return 0;
    } else {
        bool fast = res[0] == 0.0 && res[1] == 0.0;
#pragma unroll
        for (int j = 0; j < NQ; ++j) fast &= (S[j] == 0.0) && (S[NQ + j] == 0.0);
#pragma unroll
        for (int i = 2; i < NQ; ++i) {
            fast &= S[i * NQ] == 0.0;
            fast &= !(fabs(0.0 - dtl * S[i * NQ + 1]) > 1.0);  // no swap at k = 1
        }
        // decoupled directions?
        bool split = DIM > 1;
#pragma unroll
        for (int a = 0; a < NB; ++a)
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (a / NM != c / NM) split &= S[(2 + a) * NQ + (2 + c)] == 0.0;
        if constexpr (DIM > 1 && NB > 6) {
            if (!split) return 0;  // coupled 2(L+1) block too large for registers
        }
        if (!fast) return 0;
        double xm[NB];
        bool ok = true;
        if (DIM == 1 || split) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double A[NM][NM], b[NM], x[NM];
#pragma unroll
                for (int a = 0; a < NM; ++a) {
#pragma unroll
                    for (int c = 0; c < NM; ++c) {
                        const int i = 2 + d * NM + a, j = 2 + d * NM + c;
                        A[a][c] = (i == j ? 1.0 : 0.0) - dtl * S[i * NQ + j];
                        ok &= isfinite(A[a][c]);
                    }
                    b[a] = -res[2 + d * NM + a];
                }
                ok &= gepp_regs<NM>(A, b, x);
#pragma unroll
                for (int a = 0; a < NM; ++a) xm[d * NM + a] = x[a];
            }
        } else {
            if constexpr (NB <= 6) {
                double A[NB][NB], b[NB], x[NB];
#pragma unroll
                for (int a = 0; a < NB; ++a) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) {
                        A[a][c] = (a == c ? 1.0 : 0.0) - dtl * S[(2 + a) * NQ + (2 + c)];
                        ok &= isfinite(A[a][c]);
                    }
                    b[a] = -res[2 + a];
                }
                ok &= gepp_regs<NB>(A, b, x);
#pragma unroll
                for (int a = 0; a < NB; ++a) xm[a] = x[a];
            }
        }
        if (!ok || !isfinite(dtl)) return 0;
#pragma unroll
        for (int a = 0; a < NB; ++a) q[2 + a] += xm[a];
        return 1;
    }
}

// iters (optional): Newton updates applied (0 when the first residual is below
// the tolerance, so that q is returned unchanged).  Returns 1 when the
// iteration hit 15 updates, else 0.  GENERIC = false: the generic path is not
// compiled in; where an update needs it the function returns -1 and q / aux
// are left part-way (the caller discards them and defers the cell).
template <class M, bool GENERIC = true>
__device__ __forceinline__ int newton_cell(double dtl, double* q, double* aux, const double* p, int* iters = nullptr) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const double X0[3] = {0.0, 0.0, 0.0};
    double q_old[NQ], res[NQ];
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
        const auto dSdQ = M::source_jacobian_wrt_variables(q, aux, p);
        const auto dSdA = M::source_jacobian_wrt_aux_variables(q, aux, p);
        bool need = false;
#pragma unroll
        for (int e = 0; e < NQ * NA; ++e) need |= (dSdA[e] != 0.0);
#pragma unroll
        for (int i = 0; i < NQ; ++i) need |= !isfinite(q[i]);
        if (!need && newton_fast<M>(dtl, q, res, dSdQ)) continue;
        if constexpr (!GENERIC) {
            return -1;
        } else {
            // generic path: the reference's matrix and GEPP, in local memory
            double dAdQ[NA * NQ];
#pragma unroll
            for (int e = 0; e < NA * NQ; ++e) dAdQ[e] = 0.0;
            if constexpr (HasAuxJacobian<M>::value) {
                auto r = M::update_aux_variables_jacobian_wrt_variables(q, aux, p);
#pragma unroll
                for (int e = 0; e < NA * NQ; ++e) dAdQ[e] = r[e];
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
            double J[NQ * NQ], bv[NQ], xv[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i)
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    double term = dSdQ[i * NQ + j];
#pragma unroll
                    for (int k = 0; k < NA; ++k) term += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                    J[i * NQ + j] = (i == j ? 1.0 : 0.0) - dtl * term;
                }
#pragma unroll
            for (int i = 0; i < NQ; ++i) bv[i] = -res[i];
            if (!gepp_full<NQ>(J, bv, xv)) break;
#pragma unroll
            for (int i = 0; i < NQ; ++i) q[i] += xv[i];
        }
    }
    if (iters) *iters = iter;
    return iter >= 15 ? 1 : 0;
}

enum FinalizeFlags {
    FIN_PRE = 1,     // constraints after the transport update (MUSCLSolver.hpp:153)
    FIN_SOURCE = 2,  // implicit source over dt_src (SourceStep::Solve), then constraints if FIN_PRE
    FIN_POST = 4,    // constraints of PostStep (VirtualSolver.hpp:128-150)
    FIN_DT = 8,      // CFL ratio + per-instance minimum
    FIN_WRITE = 16,  // store the state / aux back
};

// One cell of the finalize step: constraints, source, constraints, store,
// CFL ratio (into ratio).  GENERIC = false: returns -1 without storing
// anything when the Newton iteration needs the generic full-size GEPP.
// GATHER: the cell's state is the last SSP stage's result, formed here from
// the face contributions (gather_final_state) instead of read from x.
template <class M, class N, bool GENERIC, bool GATHER = false>
__device__ __forceinline__ int finalize_cell(const MeshDev& m, int c, int I, double* __restrict__ x,
                                             double* __restrict__ aux, const double* p, const StepDev& sd,
                                             const double* __restrict__ dt_src, int flags, double& ratio,
                                             const FinalGather* fg = nullptr) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, DIM = M::dimension;
    const int C = m.C;
    double q[NQ], a[NA];
    if constexpr (GATHER) gather_final_state<M>(m, c, I, *fg, x, q);
    else load_q<NQ>(x, C, c, q);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    if (flags & FIN_PRE) constrain<M>(q, a, p);
    if (flags & FIN_SOURCE) {
        const int rc = newton_cell<M, GENERIC>(dt_src[I], q, a, p);
        if constexpr (!GENERIC) {
            if (rc < 0) return -1;
        }
        if (rc > 0) atomicAdd(&sd.diag[2], 1);
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
            auto rr = N::local_max_abs_eigenvalue(q, a, p, n);
            if (rr[0] > eig) eig = rr[0];
        }
        if (!(eig < 1e-14)) {
            const double rcv = m.rc[c];
            // a NaN ratio never wins a "<" comparison (VirtualSolver.hpp:342)
            if (rcv < DBL_MAX) {
                const double v = rcv / eig;
                if (v < ratio) ratio = v;
            }
        }
    }
    return 0;
}

// Appends the cells with defer set to sd.fallback (warp-aggregated, so runs
// of consecutive cells stay together).  All lanes of the warp call it.
__device__ __forceinline__ void defer_append(const StepDev& sd, bool defer, int c) {
    const unsigned dm = __ballot_sync(0xffffffffu, defer);
    if (dm) {
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == 0) base = atomicAdd(sd.n_fallback, __popc(dm));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (defer) sd.fallback[base + __popc(dm & ((1u << lane) - 1u))] = c;
    }
}

// The block's CFL ratios into the per-instance minimum sd.ratio (I < 0: no
// ratio).  Ratios are positive, so their bit patterns order like the values
// and an integer atomicMin is exact (and order-free).  Warps whose lanes
// share one instance reduce first; the block then issues one atomic per run
// of warps with the same instance.  All threads of the block call it.
__device__ __forceinline__ void block_ratio_min(const StepDev& sd, int I, double ratio) {
    unsigned long long v = (unsigned long long)__double_as_longlong(ratio);
    const int I0 = __shfl_sync(0xffffffffu, I, 0);
    const bool uniform = __all_sync(0xffffffffu, I == I0);
    __shared__ unsigned long long wv[32];
    __shared__ int wi[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (uniform) {
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_down_sync(0xffffffffu, v, off);
            if (o < v) v = o;
        }
        if (lane == 0) { wv[w] = v; wi[w] = I0; }
    } else {
        if (I >= 0 && v < ZSME_RATIO_NONE) atomicMin(&sd.ratio[I], v);
        if (lane == 0) wi[w] = -1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        int cur = -1;
        unsigned long long best = ZSME_RATIO_NONE;
        for (int k = 0; k < nw; ++k) {
            if (wi[k] < 0) continue;
            if (wi[k] != cur) {
                if (cur >= 0 && best < ZSME_RATIO_NONE) atomicMin(&sd.ratio[cur], best);
                cur = wi[k];
                best = ZSME_RATIO_NONE;
            }
            if (wv[k] < best) best = wv[k];
        }
        if (cur >= 0 && best < ZSME_RATIO_NONE) atomicMin(&sd.ratio[cur], best);
    }
}

// cells [c0, c0 + cn); dt_src: per-instance dt of the source step.
// The Newton iteration runs with the register fast path only; a cell whose
// update needs the generic GEPP is left untouched and appended to
// sd.fallback (warp-aggregated, so runs of consecutive cells stay together)
// for finalize_fallback_kernel.  Keeping the generic path out of this
// kernel lowers its stack and register pressure (1.29 -> 0.99 ms on the
// 1400^2 level-4 workload).
// MINB: resident blocks of 128 threads per SM the register allocation must allow (1 = no cap)
// GATHER: the kernel also performs the last SSP stage's gather (fg), so the
// stage result never round-trips through x; a deferred cell gets that result
// written to x for finalize_fallback_kernel.
template <class M, class N, int MINB, bool GATHER = false>
__global__ void __launch_bounds__(128, MINB) finalize_kernel(MeshDev m, int c0, int cn, double* __restrict__ x,
                                                       double* __restrict__ aux, const double* __restrict__ params,
                                                       StepDev sd, const double* __restrict__ dt_src, int flags,
                                                       FinalGather fg = FinalGather{}) {
    constexpr int NQ = M::n_dof_q;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = c0 + r;
    const int I = r < cn ? cell_instance(m, c) : -1;
    double ratio = DBL_MAX;
    const bool act = I >= 0 && (sd.active ? (sd.active[I] != 0) : true);
    bool defer = false;
    if (act) defer = finalize_cell<M, N, false, GATHER>(m, c, I, x, aux, params + (size_t)I * m.np, sd, dt_src,
                                                         flags, ratio, &fg) < 0;
    if constexpr (GATHER) {
        if (defer) {   // the generic path restarts from the stage result
            double q[NQ];
            gather_final_state<M>(m, c, I, fg, x, q);
#pragma unroll
            for (int i = 0; i < NQ; ++i) x[(size_t)i * m.C + c] = q[i];
        }
    }
    if (flags & FIN_SOURCE) defer_append(sd, defer, c);
    if (flags & FIN_DT) block_ratio_min(sd, I, ratio);
}

// The deferred cells of finalize_kernel, with the generic Newton path
// (grid-stride over sd.fallback[0 .. *sd.n_fallback)); their CFL ratios go
// straight to the per-instance atomic minimum, which is order-free.
template <class M, class N>
__global__ void __launch_bounds__(64) finalize_fallback_kernel(MeshDev m, double* __restrict__ x,
                                                               double* __restrict__ aux,
                                                               const double* __restrict__ params, StepDev sd,
                                                               const double* __restrict__ dt_src, int flags) {
    const int n = *sd.n_fallback;
    if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&sd.diag[6], n);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int c = sd.fallback[e];
        const int I = cell_instance(m, c);
        double ratio = DBL_MAX;
        finalize_cell<M, N, true>(m, c, I, x, aux, params + (size_t)I * m.np, sd, dt_src, flags, ratio);
        if ((flags & FIN_DT) && ratio < DBL_MAX)
            atomicMin(&sd.ratio[I], (unsigned long long)__double_as_longlong(ratio));
    }
}

}  // namespace zsme
