// Reverse-mode (discrete adjoint) kernels of the SME step.
//
// The forward step is X_{n+1} = Fin(Stages(X_n)) with, for SSP-RK(s,2),
//   W_0 = X_n,  W_{i+1} = W_i + dt/(s-1) R(W_i)        (i = 0 .. s-2)
//   X'  = (s-1)/s W_{s-1} + dt/s R(W_{s-1}) + 1/s W_0
// and Fin = clamp, implicit Newton source, clamp, clamp (finalize_kernel).
// R(W) is the transport right-hand side: the clamped copy wl = C(W) gives the
// neighbour bounds and the reconstruction base, W itself the gradient G, and
// each face state is wl_c + alpha_f * (G_c . dx_f) with the limiter's alpha_f.
//
// R'(W)^T v is applied by four kernels (after prep_kernel has recomputed the
// face states of W):
//   adj_face_kernel    per face side: the face state's adjoint g_f from the
//                      cells' mu = v / V through the flux and fluctuation
//                      Jacobians (dual numbers);
//   adj_cell_kernel    per cell: replays the forward reconstruction and its
//                      limiter branches (alpha_f, and for a ratio branch the
//                      component and the neighbour that bounded it) and maps g_f
//                      onto the cell's own w / wl and onto what it owes each
//                      neighbour (gradient stencil, limiter bound), one slot each;
//   adj_combine_kernel per cell: gathers what the neighbours owe it (through the
//                      neighbour's slot pointing back), applies the clamp's
//                      transposed Jacobian, and combines with the stage weights.
// Every sum is formed by one thread in a fixed order: the adjoint is
// deterministic (no atomics).
//
// adj_finalize_kernel replays finalize_kernel on the stored stage output X'
// and applies the transposed Jacobians of the clamps (dual numbers) and of the
// Newton source by the implicit-function theorem at the converged state,
//   mu = (I - dt dS/dQ)^-T lambda,  lambda_params += dt (dS/dparams)^T mu,
// with dS/dQ the total derivative through the aux state (aux = aux(Q)); a cell
// whose Newton loop took no update (residual below tolerance at once) is the
// identity, exactly as the forward map.  The CFL dt is a recorded constant:
// the adjoint is that of the step with the dt sequence of the forward run.
#pragma once
#include "dual.h"

// Register caps of the reverse kernels (face VJP / cell / finalize) as
// resident 128-thread blocks per SM (1 = uncapped): compile-time constants,
// chosen by measurement on the adjoint workload (SME level 1, 79k cells, 400
// steps, checkpoints every 20: every reverse kernel is one or a few waves, and
// the segment replays run beside the reverse sweep on a second stream, so
// resident blocks decide the time).  Replays plus reverse sweep per step:
// caps 4 / 4 / 2 0.285 ms; 4 / 5 / 2 0.283; 4 / 4 / 3 0.287; 3 / 3 / 2 0.308;
// 5 / 5 / 2 0.303; 6 / 6 / 2 0.327; 2 / 2 / 2 0.330.  The gradients are the
// same bit for bit under every cap.
#ifndef ZSME_ADJ_FACE_MINB
#define ZSME_ADJ_FACE_MINB 4
#endif
#ifndef ZSME_ADJ_CELL_MINB
#define ZSME_ADJ_CELL_MINB 4
#endif
#ifndef ZSME_ADJ_FIN_MINB
#define ZSME_ADJ_FIN_MINB 2
#endif

namespace zsme {

// li = J^T lo, J the Jacobian of update_variables at (q, a) (identity when the
// plugin has none).
template <template <typename> class MT>
__device__ __forceinline__ void clamp_adjoint(const double* q, const double* a, const double* p, const double* lo,
                                              double* li) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters;
    if constexpr (!HasUpdateVariables<M>::value) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) li[i] = lo[i];
    } else {
        using D = Dual<NQ>;
        D qd[NQ], ad[NA], pd[NP];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qd[i] = D::seed(q[i], i);
#pragma unroll
        for (int i = 0; i < NA; ++i) ad[i] = D(a[i]);
#pragma unroll
        for (int k = 0; k < NP; ++k) pd[k] = D(p[k]);
        const auto r = MT<D>::update_variables(qd, ad, pd, D(0.0));
#pragma unroll
        for (int j = 0; j < NQ; ++j) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NQ; ++i) s += r[i].d[j] * lo[i];
            li[j] = s;
        }
    }
}

// ---------------------------------------------------------------- faces
// gfs[side][NQ][F]: the adjoint of face state `side` (0: support[0], 1:
// support[1]), given the cells' adjoint v of R scaled by factor * dt, dt =
// *dtp; stage time *tp + frac * dt (time-dependent boundary conditions only).
template <template <typename> class MT, template <typename> class NT>
__global__ void __launch_bounds__(128) adj_face_kernel(MeshDev m, const double* __restrict__ fs,
                                                       const double* __restrict__ aux,
                                                       const double* __restrict__ params, const double* tp,
                                                       double frac, const double* dtp, double factor,
                                                       const double* __restrict__ v, double* __restrict__ gfs) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters;
    // One thread per (face, side), differentiating the numerical flux and the
    // fluctuations together (they share the hydrostatic reconstruction) in all
    // NQ directions of its side's face state.
    using D = Dual<NQ>;
    const int F = m.F, C = m.C;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)F * 2) return;
    const int f = (int)(tid >> 1);
    const int side = (int)(tid & 1);
    const int R = m.face_R[f], bc = m.face_bc[f], L = m.face_L[f];
    if (R < 0 && side == 1) return;  // a boundary face has one face state
    if (R < 0 && bc < 0) {  // no flux through this face
#pragma unroll
        for (int j = 0; j < NQ; ++j) gfs[(size_t)j * F + f] = 0.0;
        return;
    }
    const double* p = params + (size_t)face_instance(m, f) * m.np;
    const double area = m.farea[f];
    const double dt = *dtp;
    const double t = *tp + frac * dt;
    const double scale = factor * dt;
    D pd[NP], nh[3], xf[3];
#pragma unroll
    for (int k = 0; k < NP; ++k) pd[k] = D(p[k]);
    nh[0] = D(m.fn[f]);
    nh[1] = D(m.fn[F + f]);
    nh[2] = D(0.0);
    xf[0] = D(m.fc[f]);
    xf[1] = D(m.fc[F + f]);
    xf[2] = D(0.0);
    double muL[NQ], muR[NQ];
    {
        const double vL = m.vol[L];
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            muL[i] = scale * v[(size_t)i * C + L];
            if (vL > 1e-15) muL[i] /= vL;
            muR[i] = 0.0;
        }
        if (R >= 0) {
            const double vR = m.vol[R];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                muR[i] = scale * v[(size_t)i * C + R];
                if (vR > 1e-15) muR[i] /= vR;
            }
        }
    }
    {
        {
            D qL[NQ], aLc[NA], aL[NA];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                qL[i] = D(fs[(size_t)i * F + f]);
                if (side == 0) qL[i].d[i] = 1.0;
            }
#pragma unroll
            for (int i = 0; i < NA; ++i) aLc[i] = D(aux[(size_t)i * C + L]);
            double g[NQ];
            if (R >= 0) {
                D qR[NQ], aRc[NA], aR[NA];
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    qR[i] = D(fs[((size_t)NQ + i) * F + f]);
                    if (side == 1) qR[i].d[i] = 1.0;
                }
#pragma unroll
                for (int i = 0; i < NA; ++i) aRc[i] = D(aux[(size_t)i * C + R]);
                {
                    const auto ra = MT<D>::update_aux_variables(qL, aLc, pd, D(0.0), xf);
                    const auto rb = MT<D>::update_aux_variables(qR, aRc, pd, D(0.0), xf);
#pragma unroll
                    for (int i = 0; i < NA; ++i) { aL[i] = ra[i]; aR[i] = rb[i]; }
                }
                // cell L gets -(nc_L + F) A, cell R gets (F - nc_R) A
                const auto flux = NT<D>::numerical_flux(qL, qR, aL, aR, pd, nh);
                const auto nc = NT<D>::numerical_fluctuations(qL, qR, aL, aR, pd, nh);
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    double sum = 0.0;
#pragma unroll
                    for (int i = 0; i < NQ; ++i)
                        sum += (muR[i] - muL[i]) * area * flux[i].d[j] -
                               area * (muL[i] * nc[NQ + i].d[j] + muR[i] * nc[i].d[j]);
                    g[j] = sum;
                }
            } else {
                {
                    const auto ra = MT<D>::update_aux_variables(qL, aLc, pd, D(t), xf);
#pragma unroll
                    for (int i = 0; i < NA; ++i) aL[i] = ra[i];
                }
                const auto qR = MT<D>::boundary_conditions(bc, qL, aL, pd, nh, xf, D(t), D(0.0));
                D aR[NA];
                {
                    const auto rb = MT<D>::update_aux_variables(qR.data, aL, pd, D(t), xf);
#pragma unroll
                    for (int i = 0; i < NA; ++i) aR[i] = rb[i];
                }
                const auto flux = NT<D>::numerical_flux(qL, qR.data, aL, aR, pd, nh);
                const auto nc = NT<D>::numerical_fluctuations(qL, qR.data, aL, aR, pd, nh);
#pragma unroll
                for (int j = 0; j < NQ; ++j) {
                    double sum = 0.0;
#pragma unroll
                    for (int i = 0; i < NQ; ++i) sum -= muL[i] * area * (nc[NQ + i].d[j] + flux[i].d[j]);
                    g[j] = sum;
                }
            }
#pragma unroll
            for (int j = 0; j < NQ; ++j) gfs[((size_t)side * NQ + j) * F + f] = g[j];
        }
    }
}

// A boundary face's ghost state, as the face kernel forms it: qR =
// boundary_conditions(bc, qL, aux(qL)) at time t, with its aux.  With g
// non-null the adjoint instead: g[0 .. NQ) += (dqR / dqL)^T g[NQ .. 2 NQ)
// (dual numbers through update_aux_variables and boundary_conditions).
// Out of line, so that its dual arithmetic does not weigh on the caller's
// registers.
template <template <typename> class MT>
__device__ __noinline__ void ghost_state(const double* qL, const double* aLc, const double* p, const double* nh,
                                         const double* xf, double t, int bc, double* qR, double* aL, double* aR,
                                         double* g) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters;
    if (!g) {
        const auto ra = M::update_aux_variables(qL, aLc, p, t, xf);
#pragma unroll
        for (int i = 0; i < NA; ++i) aL[i] = ra[i];
        const auto qb = M::boundary_conditions(bc, qL, aL, p, nh, xf, t, 0.0);
#pragma unroll
        for (int i = 0; i < NQ; ++i) qR[i] = qb[i];
        const auto rb = M::update_aux_variables(qR, aL, p, t, xf);
#pragma unroll
        for (int i = 0; i < NA; ++i) aR[i] = rb[i];
        return;
    }
    using D = Dual<NQ>;
    D qd[NQ], ad[NA], pd[NP], nd[3], xd[3];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qd[i] = D::seed(qL[i], i);
#pragma unroll
    for (int i = 0; i < NA; ++i) ad[i] = D(aLc[i]);
#pragma unroll
    for (int k = 0; k < NP; ++k) pd[k] = D(p[k]);
#pragma unroll
    for (int d = 0; d < 3; ++d) { nd[d] = D(nh[d]); xd[d] = D(xf[d]); }
    const auto ra = MT<D>::update_aux_variables(qd, ad, pd, D(t), xd);
    D ald[NA];
#pragma unroll
    for (int i = 0; i < NA; ++i) ald[i] = ra[i];
    const auto qb = MT<D>::boundary_conditions(bc, qd, ald, pd, nd, xd, D(t), D(0.0));
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NQ; ++i) s += g[NQ + i] * qb[i].d[j];
        g[j] += s;
    }
}

// adj_face_kernel in one reverse sweep per face, for plugins with a
// generated numerical_flux_fluct_vjp: w^T J for both face states at once,
// w the weights adj_face_kernel contracts its dual-number Jacobian with
// (flux: (mu_R - mu_L) A; fluctuations into R: -mu_R A, into L: -mu_L A;
// at a boundary face mu_R = 0 and the fluctuations into the ghost count for
// nothing), the ghost state's dependence on the inner one pulled back by
// ghost_state.
template <template <typename> class MT, template <typename> class NT>
__global__ void __launch_bounds__(128, ZSME_ADJ_FACE_MINB) adj_face_vjp_kernel(MeshDev m, const double* __restrict__ fs,
                                                           const double* __restrict__ aux,
                                                           const double* __restrict__ params, const double* tp,
                                                           double frac, const double* dtp, double factor,
                                                           const double* __restrict__ v, double* __restrict__ gfs) {
    using M = MT<double>;
    using N = NT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int F = m.F, C = m.C;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int R = m.face_R[f], L = m.face_L[f], bc = m.face_bc[f];
    if (R < 0 && bc < 0) {  // no flux through this face
#pragma unroll
        for (int j = 0; j < NQ; ++j) gfs[(size_t)j * F + f] = 0.0;
        return;
    }
    const double* p = params + (size_t)face_instance(m, f) * m.np;
    const double area = m.farea[f];
    const double dt = *dtp;
    const double scale = factor * dt;
    const double vL = m.vol[L], vR = R >= 0 ? m.vol[R] : 0.0;
    double w[3 * NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        double muL = scale * v[(size_t)i * C + L];
        if (vL > 1e-15) muL /= vL;
        double muR = 0.0;
        if (R >= 0) {
            muR = scale * v[(size_t)i * C + R];
            if (vR > 1e-15) muR /= vR;
        }
        w[i] = (muR - muL) * area;
        w[NQ + i] = -(area * muR);
        w[2 * NQ + i] = -(area * muL);
    }
    const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
    const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
    double qL[NQ], qR[NQ], aL[NA], aR[NA], aLc[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qL[i] = fs[(size_t)i * F + f];
#pragma unroll
    for (int i = 0; i < NA; ++i) aLc[i] = aux[(size_t)i * C + L];
    const double t = *tp + frac * dt;
    if (R >= 0) {
        double aRc[NA];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qR[i] = fs[((size_t)NQ + i) * F + f];
#pragma unroll
        for (int i = 0; i < NA; ++i) aRc[i] = aux[(size_t)i * C + R];
        const auto ra = M::update_aux_variables(qL, aLc, p, 0.0, xf);
        const auto rb = M::update_aux_variables(qR, aRc, p, 0.0, xf);
#pragma unroll
        for (int i = 0; i < NA; ++i) { aL[i] = ra[i]; aR[i] = rb[i]; }
    } else {
        ghost_state<MT>(qL, aLc, p, nh, xf, t, bc, qR, aL, aR, nullptr);
    }
    double g[2 * NQ];
    N::numerical_flux_fluct_vjp(qL, qR, aL, aR, p, nh, w, g);
    if (R < 0) ghost_state<MT>(qL, aLc, p, nh, xf, t, bc, qR, aL, aR, g);
#pragma unroll
    for (int j = 0; j < NQ; ++j) gfs[(size_t)j * F + f] = g[j];
    if (R >= 0) {
#pragma unroll
        for (int j = 0; j < NQ; ++j) gfs[((size_t)NQ + j) * F + f] = g[NQ + j];
    }
}

// ---------------------------------------------------------------- cells
// own_w / own_wl [NQ][C]: adjoint of the cell's raw / clamped stage state
// from its own face states; out_w / out_wl [K][NQ][C]: what the cell owes
// the neighbour of each slot (raw: gradient stencil; clamped: limiter bound).
template <template <typename> class MT, int KM>
__global__ void __launch_bounds__(128, ZSME_ADJ_CELL_MINB) adj_cell_kernel(MeshDev m, Opts o, const double* __restrict__ w,
                                                       const double* __restrict__ wl,
                                                       const double* __restrict__ params,
                                                       const double* __restrict__ gfs, double* __restrict__ own_w,
                                                       double* __restrict__ own_wl, double* __restrict__ out_w,
                                                       double* __restrict__ out_wl,
                                                       const double* __restrict__ dec = nullptr) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            out_w[((size_t)k * NQ + i) * C + c] = 0.0;
            out_wl[((size_t)k * NQ + i) * C + c] = 0.0;
        }
    double ow[NQ], owl[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) { ow[i] = 0.0; owl[i] = 0.0; }
    int nb[KM], ff[KM], sd[KM];
    double dx[KM][DIM];
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        nb[k] = -2;
        ff[k] = -1;
        sd[k] = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) dx[k][d] = 0.0;
        if (k < K) {
            nb[k] = m.slot_nbr[k * C + c];
            ff[k] = m.slot_face[k * C + c];
            sd[k] = meta_isL(m.slot_meta[k * C + c]) ? 0 : 1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) dx[k][d] = m.slot_dx[((size_t)k * 2 + d) * C + c];
        }
    }
    if (o.order < 2) {  // piecewise constant: every face state is C(w_c)
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (ff[k] < 0) continue;
#pragma unroll
            for (int i = 0; i < NQ; ++i)
                owl[i] += gfs[((size_t)sd[k] * NQ + i) * F + ff[k]];
        }
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            own_w[(size_t)i * C + c] = 0.0;
            own_wl[(size_t)i * C + c] = owl[i];
        }
        return;
    }
    // the forward gradient (prep_kernel, same operations)
    // and its limiter, as the replay recorded them (prep_tape_kernel), or
    // recomputed from the stage state
    double g[NQ * DIM];
    double al[KM], dqs[KM];
    int js[KM], ks[KM];
    if (dec) {
#pragma unroll
        for (int i = 0; i < NQ * DIM; ++i) g[i] = dec[(size_t)i * C + c];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            al[k] = 1.0;
            dqs[k] = 1.0;
            js[k] = -1;
            ks[k] = -1;
            if (k < K) {
                al[k] = dec[((size_t)NQ * DIM + k) * C + c];
                dqs[k] = dec[((size_t)NQ * DIM + K + k) * C + c];
                const int jk = (int)dec[((size_t)NQ * DIM + 2 * K + k) * C + c];
                js[k] = (jk & 255) - 1;
                ks[k] = (jk >> 8) - 1;
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < NQ * DIM; ++i) g[i] = 0.0;
        if (o.gradient == 1) {
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                if (nb[k] < 0) continue;
                double wk[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[((size_t)k * 2 + d) * C + c];
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const double du = w[(size_t)i * C + nb[k]] - w[(size_t)i * C + c];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[i * DIM + d] += wk[d] * du;
                }
            }
        } else {
            const int ord = m.order[c];
            for (int j = 0; j < K; ++j) {
                const int k = (ord >> (2 * j)) & 3;
                const int f = m.slot_face[k * C + c];
                if (f < 0) continue;
                const int meta = m.slot_meta[k * C + c];
                const int n = m.slot_nbr[k * C + c];
                const double Nf[2] = {m.fnr[f], m.fnr[F + f]};
                if (n >= 0) {
                    const bool isL = meta_isL(meta);
#pragma unroll
                    for (int i = 0; i < NQ; ++i) {
                        const double qc = w[(size_t)i * C + c], qn = w[(size_t)i * C + n];
                        const double fv = 0.5 * (isL ? (qc + qn) : (qn + qc));
#pragma unroll
                        for (int d = 0; d < DIM; ++d) {
                            const double vv = fv * Nf[d];
                            if (isL) g[i * DIM + d] += vv;
                            else g[i * DIM + d] -= vv;
                        }
                    }
                } else if (meta_bc(meta) >= 0) {
                    double qg[NQ];
                    load_q<NQ>(w, C, c, qg);
                    const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
                    const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
                    const auto qb = M::boundary_conditions(meta_bc(meta), qg, (const double*)nullptr, p, nh, xf, 0.0, 0.0);
#pragma unroll
                    for (int i = 0; i < NQ; ++i)
#pragma unroll
                        for (int d = 0; d < DIM; ++d) g[i * DIM + d] += qb[i] * Nf[d];
                }
            }
            const double vol = m.vol[c];
            if (vol > 1e-15) {
#pragma unroll
                for (int i = 0; i < NQ * DIM; ++i) g[i] /= vol;
            }
        }
        // the forward limiter, remembering which branch set each face's alpha
#pragma unroll
        for (int k = 0; k < KM; ++k) { al[k] = 1.0; dqs[k] = 1.0; js[k] = -1; ks[k] = -1; }
        if (o.limiter) {
            bool vac = false;
            if (NQ > 1) {
                double mnh = wl[C + c];
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    if (nb[k] < 0) continue;
                    const double vv = wl[(size_t)C + nb[k]];
                    if (vv < mnh) mnh = vv;
                }
                vac = mnh < 1e-2;
            }
            if (vac) {
#pragma unroll
                for (int k = 0; k < KM; ++k) al[k] = 0.0;
            } else {
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const double q = wl[(size_t)i * C + c];
                    double mn = q, mx = q;
                    int kmn = -1, kmx = -1;
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        if (nb[k] < 0) continue;
                        const double vv = wl[(size_t)i * C + nb[k]];
                        if (vv < mn) { mn = vv; kmn = k; }
                        if (vv > mx) { mx = vv; kmx = k; }
                    }
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        if (ff[k] < 0) continue;
                        double d = 0.0;
#pragma unroll
                        for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
                        const double qfu = q + d;
                        const double dq = qfu - q;
                        double a = 1.0;
                        bool ratio = false;
                        if (!(fabs(dq) < 1e-12)) {
                            if (dq > 0) {
                                const double rr = mx - q;
                                if (mx > q) {
                                    if (!(rr >= dq)) { a = fmin(1.0, rr / dq); ratio = true; }
                                } else {
                                    a = 0.0;
                                }
                            } else {
                                const double rr = mn - q;
                                if (mn < q) {
                                    if (!(rr <= dq)) { a = fmin(1.0, rr / dq); ratio = true; }
                                } else {
                                    a = 0.0;
                                }
                            }
                        }
                        if (a < al[k]) {
                            al[k] = a;
                            js[k] = ratio ? i : -1;
                            ks[k] = dq > 0 ? kmx : kmn;
                            dqs[k] = dq;
                        }
                    }
                }
            }
        }
    }
    // face states q_f = wl_c + alpha_f (G_c . dx_f): adjoints
    double gam[NQ * DIM];
#pragma unroll
    for (int i = 0; i < NQ * DIM; ++i) gam[i] = 0.0;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        if (ff[k] < 0) continue;
        double abar = 0.0;
        double gk[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            gk[i] = gfs[((size_t)sd[k] * NQ + i) * F + ff[k]];
            double d = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
            owl[i] += gk[i];
            abar += gk[i] * d;
#pragma unroll
            for (int e = 0; e < DIM; ++e) gam[i * DIM + e] += al[k] * gk[i] * dx[k][e];
        }
        if (js[k] >= 0 && ks[k] >= 0) {
            // alpha = (bound - q_j) / dq_j with dq_j = G_j . dx
            const int j = js[k];
            const double fac = abar / dqs[k];
            out_wl[((size_t)ks[k] * NQ + j) * C + c] += fac;
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                if (i != j) continue;
                owl[i] -= fac;
#pragma unroll
                for (int e = 0; e < DIM; ++e) gam[i * DIM + e] -= fac * al[k] * dx[k][e];
            }
        }
    }
    // gradient adjoints onto the raw states of the cell and its neighbours
    if (o.gradient == 1) {
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (nb[k] < 0) continue;
            double wk[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[((size_t)k * 2 + d) * C + c];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                double s = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) s += gam[i * DIM + d] * wk[d];
                ow[i] -= s;
                out_w[((size_t)k * NQ + i) * C + c] += s;
            }
        }
    } else {
        const double vol = m.vol[c];
        if (vol > 1e-15) {
#pragma unroll
            for (int i = 0; i < NQ * DIM; ++i) gam[i] /= vol;
        }
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (ff[k] < 0) continue;
            const int f = ff[k];
            const int meta = m.slot_meta[k * C + c];
            const double Nf[2] = {m.fnr[f], m.fnr[F + f]};
            if (nb[k] >= 0) {
                const double sg = meta_isL(meta) ? 0.5 : -0.5;
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    double s = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s += gam[i * DIM + d] * Nf[d];
                    ow[i] += sg * s;
                    out_w[((size_t)k * NQ + i) * C + c] += sg * s;
                }
            } else if (meta_bc(meta) >= 0) {
                constexpr int NP = M::n_parameters;
                using D = Dual<NQ>;
                D qd[NQ], pd[NP], nh[3], xf[3];
#pragma unroll
                for (int i = 0; i < NQ; ++i) qd[i] = D::seed(w[(size_t)i * C + c], i);
#pragma unroll
                for (int kk = 0; kk < NP; ++kk) pd[kk] = D(p[kk]);
                nh[0] = D(m.fn[f]);
                nh[1] = D(m.fn[F + f]);
                nh[2] = D(0.0);
                xf[0] = D(m.fc[f]);
                xf[1] = D(m.fc[F + f]);
                xf[2] = D(0.0);
                const auto qb = MT<D>::boundary_conditions(meta_bc(meta), qd, (const D*)nullptr, pd, nh, xf, D(0.0),
                                                           D(0.0));
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    double s = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) s += gam[i * DIM + d] * Nf[d];
#pragma unroll
                    for (int j = 0; j < NQ; ++j) ow[j] += qb[i].d[j] * s;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        own_w[(size_t)i * C + c] = ow[i];
        own_wl[(size_t)i * C + c] = owl[i];
    }
}

// dst = c_src * src + (own + gathered neighbour terms), the clamped part
// through the clamp's transposed Jacobian at w.
// What the last combine of a reverse step also does, where its output is the
// step's adjoint: ax_x != null makes it ax_a ax_x + 1 v (the W_0 share of X'),
// then first != null adds the seeds of the observations of step *n0 + k, one
// by one in list order (as adj_seed_seg_kernel does).
struct AdjEpilogue {
    const double* ax_x = nullptr;
    double ax_a = 0.0;
    const int* first = nullptr;
    const int* n0 = nullptr;
    int k = 0;
    const int* cell = nullptr;
    const int* comp = nullptr;
    const double* seed = nullptr;
};

template <template <typename> class MT>
__global__ void __launch_bounds__(128) adj_combine_kernel(MeshDev m, const double* __restrict__ w,
                                                          const double* __restrict__ aux,
                                                          const double* __restrict__ params,
                                                          const double* __restrict__ own_w,
                                                          const double* __restrict__ own_wl,
                                                          const double* __restrict__ out_w,
                                                          const double* __restrict__ out_wl, const double* src,
                                                          double c_src, double* dst,
                                                          AdjEpilogue ep = AdjEpilogue{}) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double lw[NQ], lwl[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        lw[i] = own_w[(size_t)i * C + c];
        lwl[i] = own_wl[(size_t)i * C + c];
    }
    for (int k = 0; k < m.K; ++k) {
        const int n = m.slot_nbr[k * C + c];
        if (n < 0) continue;
        const int ns = meta_nslot(m.slot_meta[k * C + c]);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            lw[i] += out_w[((size_t)ns * NQ + i) * C + n];
            lwl[i] += out_wl[((size_t)ns * NQ + i) * C + n];
        }
    }
    double q[NQ], a[NA], tl[NQ];
    load_q<NQ>(w, C, c, q);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    clamp_adjoint<MT>(q, a, params + (size_t)cell_instance(m, c) * m.np, lwl, tl);
    int j0 = 0, j1 = 0;
    if (ep.first) {
        const int n = *ep.n0 + ep.k;
        j0 = ep.first[n];
        j1 = ep.first[n + 1];
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        double v = c_src * src[(size_t)i * C + c] + lw[i] + tl[i];
        if (ep.ax_x) v = ep.ax_a * ep.ax_x[(size_t)i * C + c] + 1.0 * v;
        for (int j = j0; j < j1; ++j)
            if (ep.cell[j] == c && ep.comp[j] == i) v += ep.seed[j];
        dst[(size_t)i * C + c] = v;
    }
}

// --------------------------------------------------------------- finalize
// lam_in = adjoint of the stage output X' given lam_out, the adjoint of the
// step's result; lp_part[NP][gridDim.x] += this step's parameter adjoint summed
// over each block's cells (blockDim.x = 128, fixed-order tree); the partials
// are reduced over the blocks once, after the last step.
// One cell of adj_finalize_kernel; lp[k * lp_stride] receives the cell's
// parameter adjoint k.
template <template <typename> class MT>
__device__ __forceinline__ void adj_finalize_cell(const MeshDev& m, int c, const double* __restrict__ xp,
                                                  const double* __restrict__ aux, const double* __restrict__ params,
                                                  double dt, int flags, const double* __restrict__ lam_out,
                                                  double* __restrict__ lam_in, double* lp, int lp_stride) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters;
    const int C = m.C;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    // forward replay: q0 -(pre)-> q1 -(newton)-> q2 -(pre)-> q3 -(post)-> out
    double q0[NQ], a0[NA], q2[NQ], a2[NA], q3[NQ], a3[NA];
    load_q<NQ>(xp, C, c, q0);
#pragma unroll
    for (int i = 0; i < NA; ++i) a0[i] = aux[(size_t)i * C + c];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q2[i] = q0[i];
#pragma unroll
    for (int i = 0; i < NA; ++i) a2[i] = a0[i];
    if (flags & FIN_PRE) constrain<M>(q2, a2, p);
    int iters = 0;
    if (flags & FIN_SOURCE) newton_cell<M>(dt, q2, a2, p, &iters);
#pragma unroll
    for (int i = 0; i < NQ; ++i) q3[i] = q2[i];
#pragma unroll
    for (int i = 0; i < NA; ++i) a3[i] = a2[i];
    if ((flags & FIN_SOURCE) && (flags & FIN_PRE)) constrain<M>(q3, a3, p);
    double lam[NQ], tmp[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) lam[i] = lam_out[(size_t)i * C + c];
    if (flags & FIN_POST) {
        clamp_adjoint<MT>(q3, a3, p, lam, tmp);
#pragma unroll
        for (int i = 0; i < NQ; ++i) lam[i] = tmp[i];
    }
    if (flags & FIN_SOURCE) {
        if (flags & FIN_PRE) {
            clamp_adjoint<MT>(q2, a2, p, lam, tmp);
#pragma unroll
            for (int i = 0; i < NQ; ++i) lam[i] = tmp[i];
        }
        if (iters > 0) {
            // total derivatives of S(q, aux(q), params) at the converged state
            constexpr int ND = NQ + NP;
            using D = Dual<ND>;
            D qd[NQ], ad[NA], pd[NP];
            const D X0[3] = {D(0.0), D(0.0), D(0.0)};
#pragma unroll
            for (int i = 0; i < NQ; ++i) qd[i] = D::seed(q2[i], i);
#pragma unroll
            for (int k = 0; k < NP; ++k) pd[k] = D::seed(p[k], NQ + k);
#pragma unroll
            for (int i = 0; i < NA; ++i) ad[i] = D(a2[i]);
            {
                const auto ua = MT<D>::update_aux_variables(qd, ad, pd, D(0.0), X0);
#pragma unroll
                for (int i = 0; i < NA; ++i) ad[i] = ua[i];
            }
            const auto S = MT<D>::source(qd, ad, pd, D(0.0), D(dt), X0);
            // (I - dt dS/dQ)^T mu = lam
            double JT[NQ * NQ], bv[NQ], mu[NQ];
#pragma unroll
            for (int i = 0; i < NQ; ++i)
#pragma unroll
                for (int j = 0; j < NQ; ++j) JT[j * NQ + i] = (i == j ? 1.0 : 0.0) - dt * S[i].d[j];
#pragma unroll
            for (int i = 0; i < NQ; ++i) bv[i] = lam[i];
            if (gepp_full<NQ>(JT, bv, mu)) {
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    double s = 0.0;
#pragma unroll
                    for (int i = 0; i < NQ; ++i) s += mu[i] * dt * S[i].d[NQ + k];
                    lp[k * lp_stride] = s;
                }
#pragma unroll
                for (int i = 0; i < NQ; ++i) lam[i] = mu[i];
            }
        }
    }
    if (flags & FIN_PRE) {
        clamp_adjoint<MT>(q0, a0, p, lam, tmp);
#pragma unroll
        for (int i = 0; i < NQ; ++i) lam[i] = tmp[i];
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i) lam_in[(size_t)i * C + c] = lam[i];
}

template <template <typename> class MT>
__global__ void __launch_bounds__(128, ZSME_ADJ_FIN_MINB) adj_finalize_kernel(MeshDev m, const double* __restrict__ xp,
                                                           const double* __restrict__ aux,
                                                           const double* __restrict__ params, const double* dtp,
                                                           int flags, const double* __restrict__ lam_out,
                                                           double* __restrict__ lam_in,
                                                           double* __restrict__ lp_part) {
    using M = MT<double>;
    constexpr int NQ = M::n_dof_q, NP = M::n_parameters;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ double lp_sh[NP][128];
#pragma unroll
    for (int k = 0; k < NP; ++k) lp_sh[k][threadIdx.x] = 0.0;
    const double dt = *dtp;
    if (c < C) {
        if (dt > 0.0) {
            adj_finalize_cell<MT>(m, c, xp, aux, params, dt, flags, lam_out, lam_in, &lp_sh[0][0] + threadIdx.x, 128);
        } else {  // a step after t_end changed nothing
#pragma unroll
            for (int i = 0; i < NQ; ++i) lam_in[(size_t)i * C + c] = lam_out[(size_t)i * C + c];
        }
    }
    __syncthreads();
    for (int h = 64; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
#pragma unroll
            for (int k = 0; k < NP; ++k) lp_sh[k][threadIdx.x] += lp_sh[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)   // each block accumulates its cells' sum over the steps
#pragma unroll
        for (int k = 0; k < NP; ++k) lp_part[(size_t)k * gridDim.x + blockIdx.x] += lp_sh[k][0];
}

// ------------------------------------------------------------- small ones
// lp_total[k] += sum of the nb block partials lp_part[k][.] (one block per
// parameter, fixed order: deterministic)
static __global__ void __launch_bounds__(256) adj_param_reduce_kernel(const double* __restrict__ lp_part, int nb,
                                                                      double* __restrict__ lp_total) {
    __shared__ double sh[256];
    const int k = blockIdx.x;
    double s = 0.0;
    for (int c = threadIdx.x; c < nb; c += blockDim.x) s += lp_part[(size_t)k * nb + c];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) lp_total[k] += sh[0];
}

// oval[j] = x[comp_j][cell_j] (device cell numbering)
static __global__ void obs_value_kernel(int n, const int* __restrict__ cell, const int* __restrict__ comp,
                                        const double* __restrict__ x, int C, double* __restrict__ oval) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) oval[j] = x[(size_t)comp[j] * C + cell[j]];
}

// lam[comp_j][cell_j] += seed_j for the n observations, one after the other
static __global__ void adj_seed_kernel(int n, const int* __restrict__ cell, const int* __restrict__ comp,
                                       const double* __restrict__ seed, int C, double* __restrict__ lam) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int j = 0; j < n; ++j) lam[(size_t)comp[j] * C + cell[j]] += seed[j];
}

// the seeds of the observations of step *n0 + k (first: per-step CSR offsets)
static __global__ void adj_seed_seg_kernel(const int* __restrict__ first, const int* __restrict__ n0, int k,
                                           const int* __restrict__ cell, const int* __restrict__ comp,
                                           const double* __restrict__ seed, int C, double* __restrict__ lam) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int n = *n0 + k;
    for (int j = first[n]; j < first[n + 1]; ++j) lam[(size_t)comp[j] * C + cell[j]] += seed[j];
}

// y = a x + b y over n values
static __global__ void axpby_kernel(long long n, double a, const double* __restrict__ x, double b, double* y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a * x[i] + b * y[i];
}

}  // namespace zsme
