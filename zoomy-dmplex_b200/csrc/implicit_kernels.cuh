// Kernels of the fully implicit strategy (SolverStrategies.hpp:133-195): BDF
// in time, the residual F(t, X, Xdot) = Xdot - S(X) - R(X) of
// IFunctionWrapper (the transport right-hand side R comes from the ordinary
// prep / face / gather kernels in MODE_RHS, the source S is the IMEX
// strategy's implicit source), and the preconditioning matrix of
// ModularSolver::FormImplicitJacobian (ModularSolver.hpp:238-371): per cell
// a I - dS/dQ (the identity times a in cells drier than 1e-4) plus the
// forward-difference Jacobians of each face's flux and fluctuations at the
// cell states, scaled by area / volume.  Matrix entries are summed in the
// reference's assembly order (all source blocks, then the faces in increasing
// original face id), so the blocks agree with the CPU restatement bit for
// bit.  The Newton-Krylov iteration around them runs on the host
// (solver.cuh); the vector kernels here serve its GMRES.
#pragma once
#include "imex_kernels.cuh"

namespace zsme {

namespace implicit_fd {
constexpr double eps = 1e-7;       // ComputeFaceJacobian_FD / ComputeBoundaryJacobian_FD step
constexpr double dry_jacobian = 1e-4;
}  // namespace implicit_fd

// f = (Xdot - S(y)) - R, Xdot = xdot[id] when given, else
// (c0 y + c1 xn + c2 xnm1) / h (the BDF derivative of the step), the
// coefficients c0, c1, c2, h from device memory (coef) when given
struct BdfTerms {
    const double* xdot;
    const double* xn;
    const double* xnm1;
    double c0, c1, c2, h;
    const double* coef;
};

template <class M>
__global__ void __launch_bounds__(128) imp_residual_kernel(MeshDev m, const double* __restrict__ y,
                                                           const double* __restrict__ aux,
                                                           const double* __restrict__ params,
                                                           const double* __restrict__ R, BdfTerms b,
                                                           double* __restrict__ f) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    double q[NQ], a[NA], S[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = y[(size_t)i * C + c];
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    imex_source_cell<M>(q, a, p, S);
    const double c0 = b.coef ? b.coef[0] : b.c0, c1 = b.coef ? b.coef[1] : b.c1;
    const double c2 = b.coef ? b.coef[2] : b.c2, h = b.coef ? b.coef[3] : b.h;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const size_t id = (size_t)i * C + c;
        const double xd = b.xdot ? b.xdot[id] : (c0 * q[i] + c1 * b.xn[id] + c2 * b.xnm1[id]) / h;
        f[id] = (xd - S[i]) - R[id];
    }
}

// The four forward-difference blocks of one interior face (ComputeFaceJacobian_FD,
// ModularSolver.hpp:130-185) or the one block of a boundary face with a
// condition (ComputeBoundaryJacobian_FD, :187-236), each scaled by area /
// volume of its row's cell.  fj [F][4][NQ][NQ]: LL, LR, RL, RR.  Column j of
// every block comes from one perturbed evaluation, so no block is held whole.
template <class M, class N>
__global__ void __launch_bounds__(128) imp_face_jac_kernel(MeshDev m, const double* __restrict__ xl,
                                                           const double* __restrict__ al,
                                                           const double* __restrict__ params, double t,
                                                           double* __restrict__ fj) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, Q2 = NQ * NQ;
    const int F = m.F, C = m.C;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    double* out = fj + (size_t)f * 4 * Q2;
    const int L = m.face_L[f], R = m.face_R[f], bc = m.face_bc[f];
    const double area = m.farea[f];
    const bool used = area > 1e-15 && (R >= 0 || bc >= 0);
    if (!used) {
        for (int e = 0; e < 4 * Q2; ++e) out[e] = 0.0;
        return;
    }
    const double* p = params + (size_t)face_instance(m, f) * m.np;
    const double X0[3] = {0.0, 0.0, 0.0};
    const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
    const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
    const double eps = implicit_fd::eps;
    double qL[NQ], aL[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qL[i] = xl[(size_t)i * C + L];
#pragma unroll
    for (int i = 0; i < NA; ++i) aL[i] = al[(size_t)i * C + L];
    const double fL = area / m.vol[L];
    if (R >= 0) {
        double qR[NQ], aR[NA];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qR[i] = xl[(size_t)i * C + R];
#pragma unroll
        for (int i = 0; i < NA; ++i) aR[i] = al[(size_t)i * C + R];
        const double fR = area / m.vol[R];
        const auto Fb = N::numerical_flux(qL, qR, aL, aR, p, nh);
        const auto NCb = N::numerical_fluctuations(qL, qR, aL, aR, p, nh);
        for (int side = 0; side < 2; ++side) {
            // side 0 perturbs the left state (columns of LL and RL), side 1 the right (LR and RR)
            double* Jrow0 = out + (side == 0 ? 0 : 1) * Q2;   // LL or LR, rows of L
            double* Jrow1 = out + (side == 0 ? 2 : 3) * Q2;   // RL or RR, rows of R
            for (int j = 0; j < NQ; ++j) {
                double qp[NQ], ap[NA];
#pragma unroll
                for (int k = 0; k < NQ; ++k) qp[k] = side == 0 ? qL[k] : qR[k];
#pragma unroll
                for (int k = 0; k < NA; ++k) ap[k] = side == 0 ? aL[k] : aR[k];
                qp[j] += eps;
                if (NA > 0) {
                    const auto ra = M::update_aux_variables(qp, ap, p, 0.0, X0);
#pragma unroll
                    for (int k = 0; k < NA; ++k) ap[k] = ra[k];
                }
                const auto Fp = side == 0 ? N::numerical_flux(qp, qR, ap, aR, p, nh)
                                          : N::numerical_flux(qL, qp, aL, ap, p, nh);
                const auto NCp = side == 0 ? N::numerical_fluctuations(qp, qR, ap, aR, p, nh)
                                           : N::numerical_fluctuations(qL, qp, aL, ap, p, nh);
#pragma unroll
                for (int i = 0; i < NQ; ++i) {
                    const double dFlux = (Fp[i] - Fb[i]) / eps;
                    double j0 = 0.0, j1 = 0.0;
                    j0 += dFlux;
                    j1 -= dFlux;
                    j0 += (NCp[NQ + i] - NCb[NQ + i]) / eps;
                    j1 += (NCp[i] - NCb[i]) / eps;
                    Jrow0[i * NQ + j] = j0 * fL;
                    Jrow1[i * NQ + j] = j1 * fR;
                }
            }
        }
    } else {
        double qRb[NQ], aRb[NA];
        {
            const auto r = M::boundary_conditions(bc, qL, aL, p, nh, xf, t, 0.0);
#pragma unroll
            for (int i = 0; i < NQ; ++i) qRb[i] = r[i];
            if (NA > 0) {
                const auto ra = M::update_aux_variables(qRb, aL, p, t, xf);
#pragma unroll
                for (int k = 0; k < NA; ++k) aRb[k] = ra[k];
            }
        }
        const auto Fb = N::numerical_flux(qL, qRb, aL, aRb, p, nh);
        const auto NCb = N::numerical_fluctuations(qL, qRb, aL, aRb, p, nh);
        for (int j = 0; j < NQ; ++j) {
            double qp[NQ], ap[NA], qr[NQ], ar[NA];
#pragma unroll
            for (int k = 0; k < NQ; ++k) qp[k] = qL[k];
#pragma unroll
            for (int k = 0; k < NA; ++k) ap[k] = aL[k];
            qp[j] += eps;
            if (NA > 0) {
                const auto ra = M::update_aux_variables(qp, ap, p, t, xf);
#pragma unroll
                for (int k = 0; k < NA; ++k) ap[k] = ra[k];
            }
            {
                const auto r = M::boundary_conditions(bc, qp, ap, p, nh, xf, t, 0.0);
#pragma unroll
                for (int k = 0; k < NQ; ++k) qr[k] = r[k];
            }
            if (NA > 0) {
                const auto ra = M::update_aux_variables(qr, ap, p, t, xf);
#pragma unroll
                for (int k = 0; k < NA; ++k) ar[k] = ra[k];
            }
            const auto Fp = N::numerical_flux(qp, qr, ap, ar, p, nh);
            const auto NCp = N::numerical_fluctuations(qp, qr, ap, ar, p, nh);
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                double j0 = 0.0;
                j0 += (Fp[i] - Fb[i]) / eps;
                j0 += (NCp[NQ + i] - NCb[NQ + i]) / eps;
                out[i * NQ + j] = j0 * fL;
            }
        }
        for (int e = Q2; e < 4 * Q2; ++e) out[e] = 0.0;
    }
}

// The diagonal block of cell c, [NQ*NQ][C] (entry e = i NQ + j of every cell
// contiguous over the cells): the matrix starts at zero (MatZeroEntries), the
// cell's source block is added (a I - dS/dQ - dS/dAux dAux/dQ at the clamped
// state; a I in cells drier than 1e-4), then the face blocks of the cell's
// faces in increasing original face id (LL where the cell is the face's
// first cell, RR where it is the second; faces without a condition and
// degenerate faces add nothing, as in the reference's face loop).
template <class M>
__global__ void __launch_bounds__(64) imp_cell_jac_kernel(MeshDev m, const double* __restrict__ xl,
                                                          const double* __restrict__ al,
                                                          const double* __restrict__ params, double a,
                                                          const double* __restrict__ fj, double* __restrict__ pd) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, Q2 = NQ * NQ;
    const int C = m.C, K = m.K;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    const double X0[3] = {0.0, 0.0, 0.0};
    double q[NQ], aux[NA], J[Q2];
    for (int i = 0; i < NQ; ++i) q[i] = xl[(size_t)i * C + c];
    for (int i = 0; i < NA; ++i) aux[i] = al[(size_t)i * C + c];
    if (NQ > 1 && q[1] < implicit_fd::dry_jacobian) {
        for (int e = 0; e < Q2; ++e) J[e] = 0.0;
        for (int i = 0; i < NQ; ++i) J[i * NQ + i] = a;
    } else {
        const auto dSdQ = M::source_jacobian_wrt_variables(q, aux, p);
        const auto dSdA = M::source_jacobian_wrt_aux_variables(q, aux, p);
        double dAdQ[NA * NQ + 1];
        if constexpr (HasAuxJacobian<M>::value) {
            const auto r = M::update_aux_variables_jacobian_wrt_variables(q, aux, p);
            for (int e = 0; e < NA * NQ; ++e) dAdQ[e] = r[e];
        } else {   // forward differences, SourceStep.hpp:16-53
            const auto a0 = M::update_aux_variables(q, aux, p, 0.0, X0);
            for (int j = 0; j < NQ; ++j) {
                double qp[NQ];
                for (int mm = 0; mm < NQ; ++mm) qp[mm] = q[mm];
                const double hh = 1e-7 * (fabs(q[j]) + 1e-7);
                qp[j] += hh;
                const auto a1 = M::update_aux_variables(qp, aux, p, 0.0, X0);
                for (int k = 0; k < NA; ++k) dAdQ[k * NQ + j] = (a1[k] - a0[k]) / hh;
            }
        }
        for (int i = 0; i < NQ; ++i)
            for (int j = 0; j < NQ; ++j) {
                const double val = i == j ? a : 0.0;
                double dSource = dSdQ[i * NQ + j];
                for (int k = 0; k < NA; ++k) dSource += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                J[i * NQ + j] = val - dSource;
            }
    }
    // the cell's face blocks in increasing original face id
    const double* blk[4] = {nullptr, nullptr, nullptr, nullptr};
    int nblk = 0;
    const int ord = m.order[c];
    for (int jj = 0; jj < K; ++jj) {
        const int k = (ord >> (2 * jj)) & 3;
        const int f = m.slot_face[k * C + c];
        if (f < 0) continue;
        if (m.face_R[f] < 0 && m.face_bc[f] < 0) continue;
        if (!(m.farea[f] > 1e-15)) continue;
        blk[nblk++] = fj + ((size_t)f * 4 + (m.face_L[f] == c ? 0 : 3)) * Q2;
    }
    for (int e = 0; e < Q2; ++e) {
        double acc = 0.0;
        acc += J[e];
        for (int b = 0; b < nblk; ++b) acc += blk[b][e];
        pd[(size_t)e * C + c] = acc;
    }
}

// LU factors of every diagonal block with partial pivoting (the block-Jacobi
// preconditioner of the Krylov solve): lu in the layout of pd, piv [NQ][C];
// bad[c] = 1 where a pivot is zero or not finite (that block is applied as the
// identity).
template <int NQ>
__global__ void __launch_bounds__(64) imp_block_lu_kernel(int C, const double* __restrict__ pd,
                                                          double* __restrict__ lu, int* __restrict__ piv) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double A[NQ * NQ];
    for (int e = 0; e < NQ * NQ; ++e) A[e] = pd[(size_t)e * C + c];
    int pv[NQ];
    bool ok = true;
    for (int k = 0; k < NQ; ++k) {
        int mr = k;
        double mv = fabs(A[k * NQ + k]);
        for (int i = k + 1; i < NQ; ++i) {
            const double v = fabs(A[i * NQ + k]);
            if (v > mv) { mv = v; mr = i; }
        }
        pv[k] = mr;
        if (mr != k)
            for (int j = 0; j < NQ; ++j) {
                const double tt = A[k * NQ + j];
                A[k * NQ + j] = A[mr * NQ + j];
                A[mr * NQ + j] = tt;
            }
        const double pkk = A[k * NQ + k];
        if (!(mv > 0.0) || !isfinite(pkk)) { ok = false; break; }
        for (int i = k + 1; i < NQ; ++i) {
            const double l = A[i * NQ + k] / pkk;
            A[i * NQ + k] = l;
            for (int j = k + 1; j < NQ; ++j) A[i * NQ + j] -= l * A[k * NQ + j];
        }
    }
    if (!ok) {
        for (int e = 0; e < NQ * NQ; ++e) A[e] = 0.0;
        for (int i = 0; i < NQ; ++i) { A[i * NQ + i] = 1.0; pv[i] = i; }
    }
    for (int e = 0; e < NQ * NQ; ++e) lu[(size_t)e * C + c] = A[e];
    for (int i = 0; i < NQ; ++i) piv[(size_t)i * C + c] = pv[i];
}

// z = D^-1 r per cell from the LU factors (r and z may alias)
template <int NQ>
__global__ void __launch_bounds__(128) imp_block_solve_kernel(int C, const double* __restrict__ lu,
                                                              const int* __restrict__ piv, const double* r,
                                                              double* z) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double b[NQ];
    for (int i = 0; i < NQ; ++i) b[i] = r[(size_t)i * C + c];
    for (int k = 0; k < NQ; ++k) {
        const int mr = piv[(size_t)k * C + c];
        if (mr != k) {
            const double tt = b[k];
            b[k] = b[mr];
            b[mr] = tt;
        }
        for (int i = k + 1; i < NQ; ++i) b[i] -= lu[(size_t)(i * NQ + k) * C + c] * b[k];
    }
    for (int i = NQ - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < NQ; ++j) s -= lu[(size_t)(i * NQ + j) * C + c] * b[j];
        b[i] = s / lu[(size_t)(i * NQ + i) * C + c];
    }
    for (int i = 0; i < NQ; ++i) z[(size_t)i * C + c] = b[i];
}

// UpdateState of a state: xl = the state clamped (update_variables), al = its
// aux (update_aux_variables) from the handle's aux
template <class M>
__global__ void __launch_bounds__(128) imp_update_state_kernel(MeshDev m, const double* __restrict__ y,
                                                               const double* __restrict__ aux,
                                                               const double* __restrict__ params,
                                                               double* __restrict__ xl, double* __restrict__ al) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    double q[NQ], a[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = y[(size_t)i * C + c];
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    constrain<M>(q, a, p);
#pragma unroll
    for (int i = 0; i < NQ; ++i) xl[(size_t)i * C + c] = q[i];
#pragma unroll
    for (int i = 0; i < NA; ++i) al[(size_t)i * C + c] = a[i];
}

// ------------------------------------------------------------ vector kernels
// The matrix-free Jacobian's differencing parameter from the device dot v.v:
// hv = sqrt(eps) sqrt(1 + |X|) / |v| (0 for a zero vector)
static __global__ void imp_hv_kernel(const double* __restrict__ vv, const double* __restrict__ xnorm,
                                     double* __restrict__ hv) {
    const double vn = sqrt(*vv);
    *hv = vn > 0.0 ? 1.4901161193847656e-08 * sqrt(1.0 + *xnorm) / vn : 0.0;
}
static __global__ void imp_sqrt_kernel(const double* __restrict__ in, double* __restrict__ out) { *out = sqrt(*in); }
// out = 1.0 x + hv v, hv a device scalar
static __global__ void imp_perturb_kernel(long long n, const double* __restrict__ x, const double* __restrict__ v,
                                          const double* __restrict__ hv, double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = 1.0 * x[i] + *hv * v[i];
}
// out = (ft - f0) / hv, zero when hv is zero
static __global__ void imp_diffquot_dev_kernel(long long n, const double* __restrict__ ft,
                                               const double* __restrict__ f0, const double* __restrict__ hv,
                                               double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = *hv;
    out[i] = h != 0.0 ? (ft[i] - f0[i]) / h : 0.0;
}
// out = (1.0 / sqrt(ww)) w where ww = w.w > 0 (the next Arnoldi vector)
static __global__ void imp_normalize_kernel(long long n, const double* __restrict__ ww, const double* __restrict__ w,
                                            double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double hn = sqrt(*ww);
    if (hn > 0.0) out[i] = (1.0 / hn) * w[i];
}
// out = (ft - f0) / h (the matrix-free Jacobian's difference quotient)
static __global__ void imp_diffquot_kernel(long long n, const double* __restrict__ ft, const double* __restrict__ f0,
                                           double h, double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (ft[i] - f0[i]) / h;
}
// out = a x + b y (out may alias x or y; y may be null when b = 0)
static __global__ void imp_lincomb_kernel(long long n, double a, const double* x, double b, const double* y,
                                          double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = y ? a * x[i] + b * y[i] : a * x[i];
}

// partial[k][blk] = sum over the block's entries of V_k . w, k < nk (V_k =
// V + k ld); a fixed tree per block, so the sums are deterministic
static __global__ void __launch_bounds__(256) imp_multi_dot_kernel(long long n, int nk, const double* __restrict__ V,
                                                                   long long ld, const double* __restrict__ w,
                                                                   double* __restrict__ partial) {
    // grid (nb, nk): block (b, k) takes vector k's chunk b
    __shared__ double sh[256];
    const int nb = gridDim.x, k = blockIdx.y;
    if (k >= nk) return;
    const double* v = V + (size_t)k * ld;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)nb * blockDim.x)
        s += v[i] * w[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)k * nb + blockIdx.x] = sh[0];
}
// out[k] = sum of partial[k][0 .. nb): one block of 256 threads per k, each
// thread a fixed stride of the partials, then a fixed tree (deterministic)
static __global__ void __launch_bounds__(256) imp_reduce_kernel(int nk, int nb, const double* __restrict__ partial,
                                                                double* __restrict__ out) {
    __shared__ double sh[256];
    const int k = blockIdx.x;
    if (k >= nk) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(size_t)k * nb + b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = sh[0];
}
// w -= sum_k h_k V_k (classical Gram-Schmidt projection, h on the device)
static __global__ void imp_multi_axpy_kernel(long long n, int nk, const double* __restrict__ V, long long ld,
                                             const double* __restrict__ h, double* __restrict__ w) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = w[i];
    for (int k = 0; k < nk; ++k) s -= h[k] * V[(size_t)k * ld + i];
    w[i] = s;
}
// x += sum_k y_k V_k (the Krylov update, y on the device)
static __global__ void imp_multi_add_kernel(long long n, int nk, const double* __restrict__ V, long long ld,
                                            const double* __restrict__ y, double* __restrict__ x) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = x[i];
    for (int k = 0; k < nk; ++k) s += y[k] * V[(size_t)k * ld + i];
    x[i] = s;
}

}  // namespace zsme
