// Face fluxes, each face evaluated once, and the per-cell gather.
//
// face_kernel  one thread per face: reads the two reconstructed face states
//              (face-indexed, coalesced), evaluates Numerics::numerical_flux
//              and ::numerical_fluctuations (or the boundary ghost state) and
//              stores nc_into_left*area, nc_into_right*area, flux*area
//              (TransportStep.hpp:420-552).
// gather_kernel one thread per cell: sums its faces' contributions in
//              increasing original face order -- for each face first the
//              fluctuation, then the flux, exactly the sequence of the
//              reference's face loop (TransportStep.hpp:464-466, 529-531) --
//              divides by the volume (555-560) and applies the SSP-RK(s,2)
//              stage combination of PETSc's TSSSP "rks2" in the same pass.
#pragma once

namespace zsme {

// One face's contributions (TransportStep.hpp:420-552): out[r * ostride] for
// r in [0, NQ) the fluctuation into the left cell, [NQ, 2 NQ) into the right
// cell (interior faces only), [2 NQ, 3 NQ) the flux, each times the area.
// Returns false, writing nothing, for an exterior face without a condition
// (no flux) and for a face of an inactive instance.
template <class M, class N>
__device__ __forceinline__ bool face_contrib(const MeshDev& m, int f, const double* __restrict__ fs,
                                             const double* __restrict__ aux, const double* __restrict__ params,
                                             double t_host, const double* t_dev, double stage_frac,
                                             const double* __restrict__ dt_step, const int* __restrict__ active,
                                             double* __restrict__ out, size_t ostride) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int F = m.F, C = m.C;
    const int I = face_instance(m, f);
    if (active && !active[I]) return false;
    const double* p = params + (size_t)I * m.np;
    const int R = m.face_R[f];
    const int bc = m.face_bc[f];
    if (R < 0 && bc < 0) return false;  // exterior face without a condition: no flux
    const int L = m.face_L[f];
    // stage time t0 + dt * i/(s-1) (only time-dependent BCs / aux see it)
    const double t = t_dev ? (t_dev[I] + stage_frac * (dt_step ? dt_step[I] : 0.0)) : t_host;
    const double area = m.farea[f];
    const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
    const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
    double qL[NQ], aLc[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qL[i] = fs[(size_t)i * F + f];
#pragma unroll
    for (int i = 0; i < NA; ++i) aLc[i] = aux[(size_t)i * C + L];
    double aL[NA], aR[NA];
    if (R >= 0) {
        double qR[NQ], aRc[NA];
#pragma unroll
        for (int i = 0; i < NQ; ++i) qR[i] = fs[((size_t)NQ + i) * F + f];
#pragma unroll
        for (int i = 0; i < NA; ++i) aRc[i] = aux[(size_t)i * C + R];
        {
            auto ra = M::update_aux_variables(qL, aLc, p, 0.0, xf);
            auto rb = M::update_aux_variables(qR, aRc, p, 0.0, xf);
#pragma unroll
            for (int i = 0; i < NA; ++i) { aL[i] = ra[i]; aR[i] = rb[i]; }
        }
        const auto flux = N::numerical_flux(qL, qR, aL, aR, p, nh);
        const auto nc = N::numerical_fluctuations(qL, qR, aL, aR, p, nh);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            out[i * ostride] = nc[NQ + i] * area;
            out[(NQ + i) * ostride] = nc[i] * area;
            out[(2 * NQ + i) * ostride] = flux[i] * area;
        }
    } else {
        {
            auto ra = M::update_aux_variables(qL, aLc, p, t, xf);
#pragma unroll
            for (int i = 0; i < NA; ++i) aL[i] = ra[i];
        }
        const auto qR = M::boundary_conditions(bc, qL, aL, p, nh, xf, t, 0.0);
        {
            auto rb = M::update_aux_variables(qR.data, aL, p, t, xf);
#pragma unroll
            for (int i = 0; i < NA; ++i) aR[i] = rb[i];
        }
        const auto flux = N::numerical_flux(qL, qR.data, aL, aR, p, nh);
        const auto nc = N::numerical_fluctuations(qL, qR.data, aL, aR, p, nh);
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            out[i * ostride] = nc[NQ + i] * area;
            out[(2 * NQ + i) * ostride] = flux[i] * area;
        }
    }
    return true;
}

// faces [f0, f0 + fcount)
// MINB: resident blocks per SM the register allocation must allow (1 = no cap)
template <class M, class N, int MINB>
__global__ void __launch_bounds__(128, MINB) face_kernel(MeshDev m, int f0, int fcount, const double* __restrict__ fs,
                                                   const double* __restrict__ aux,
                                                   const double* __restrict__ params, double t_host,
                                                   const double* t_dev, double stage_frac,
                                                   const double* __restrict__ dt_step, double* __restrict__ fb,
                                                   const int* __restrict__ active) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= fcount) return;
    const int f = f0 + r;
    face_contrib<M, N>(m, f, fs, aux, params, t_host, t_dev, stage_frac, dt_step, active, fb + f, (size_t)m.F);
}

// Division by the volume (TransportStep.hpp:555-560) and the SSP-RK(s,2)
// stage combination of PETSc's TSSSP "rks2" for cell c of instance I, whose
// summed face contributions are acc.
template <class M>
__device__ __forceinline__ void stage_update(const MeshDev& m, const Opts& o, int c, int I, double* acc, int mode,
                                             const double* x_in, double* x_out, double* base,
                                             const double* __restrict__ dt_step, const double* __restrict__ aux,
                                             const double* __restrict__ params, double* __restrict__ xl_out) {
    constexpr int NQ = M::n_dof_q;
    const int C = m.C;
    const double v = m.vol[c];
    if (v > 1e-15) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) acc[i] /= v;
    }
    const double h = dt_step ? dt_step[I] : 0.0;
    const int s = o.stages;
    switch (mode) {
        case MODE_RHS:
#pragma unroll
            for (int i = 0; i < NQ; ++i) x_out[(size_t)i * C + c] = acc[i];
            break;
        case MODE_FIRST:    // w = x + dt/(s-1) F
        case MODE_MID: {    // w += dt/(s-1) F (in place)
            const double a = h / (s - 1.);
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                acc[i] = x_in[(size_t)i * C + c] + a * acc[i];
                x_out[(size_t)i * C + c] = acc[i];
            }
            if (xl_out) {   // the next stage's clamped copy
                constexpr int NA = M::n_dof_qaux;
                double an[NA];
#pragma unroll
                for (int i = 0; i < NA; ++i) an[i] = aux[(size_t)i * C + c];
                clamp_q<M>(acc, an, params + (size_t)I * m.np);
#pragma unroll
                for (int i = 0; i < NQ; ++i) xl_out[(size_t)i * C + c] = acc[i];
            }
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

// The last SSP stage's gather, for finalize_kernel to fuse: the face
// contributions, the stage state W_{s-1} and the step's per-instance dt.
struct FinalGather {
    const double* fb;
    const double* w;
    const double* dt_step;
    int stages;
};

// Cell c's state after the last SSP stage (gather_kernel's MODE_FINAL
// value, the same operations in the same order) into q, from the step's
// start state x; nothing is written.
template <class M>
__device__ __forceinline__ void gather_final_state(const MeshDev& m, int c, int I, const FinalGather& fg,
                                                   const double* __restrict__ x, double* q) {
    constexpr int NQ = M::n_dof_q;
    const int C = m.C, F = m.F;
    const double* __restrict__ fb = fg.fb;
    double acc[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
    const int ord = m.order[c];
    for (int j = 0; j < m.K; ++j) {
        const int k = (ord >> (2 * j)) & 3;
        const int f = m.slot_face[k * C + c];
        if (f < 0) continue;
        const int meta = m.slot_meta[k * C + c];
        if (m.slot_nbr[k * C + c] < 0 && meta_bc(meta) < 0) continue;
        if (meta_isL(meta)) {
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[(size_t)i * F + f];
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[((size_t)2 * NQ + i) * F + f];
        } else {
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[((size_t)NQ + i) * F + f];
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] += fb[((size_t)2 * NQ + i) * F + f];
        }
    }
    const double v = m.vol[c];
    if (v > 1e-15) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) acc[i] /= v;
    }
    const int s = fg.stages;
    const double h = fg.dt_step[I];
    const double al = (s - 1.) / s, be = h / s, ga = 1. / s;
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const size_t id = (size_t)i * C + c;
        q[i] = al * fg.w[id] + be * acc[i] + ga * x[id];
    }
}

// cells [c0, c0 + cn)
template <class M>
__global__ void __launch_bounds__(128) gather_kernel(MeshDev m, Opts o, int c0, int cn,
                                                     const double* __restrict__ fb, int mode, const double* x_in,
                                                     double* x_out, double* base, const double* __restrict__ dt_step,
                                                     const int* __restrict__ active, const double* __restrict__ aux,
                                                     const double* __restrict__ params, double* __restrict__ xl_out) {
    constexpr int NQ = M::n_dof_q;
    const int C = m.C, F = m.F;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    double acc[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
    const int ord = m.order[c];
    for (int j = 0; j < m.K; ++j) {
        const int k = (ord >> (2 * j)) & 3;
        const int f = m.slot_face[k * C + c];
        if (f < 0) continue;
        const int meta = m.slot_meta[k * C + c];
        if (m.slot_nbr[k * C + c] < 0 && meta_bc(meta) < 0) continue;
        if (meta_isL(meta)) {
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[(size_t)i * F + f];
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[((size_t)2 * NQ + i) * F + f];
        } else {
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] -= fb[((size_t)NQ + i) * F + f];
#pragma unroll
            for (int i = 0; i < NQ; ++i) acc[i] += fb[((size_t)2 * NQ + i) * F + f];
        }
    }
    stage_update<M>(m, o, c, I, acc, mode, x_in, x_out, base, dt_step, aux, params, xl_out);
}

// ------------------------------------------------------- fused face + gather
// Device view of FaceTiles (prepared_mesh.h).
struct TilesDev {
    const int* cell_off;  // [n + 1]
    const int* face_off;  // [n + 1]
    const int* in_off;    // [n + 1]
    const int* in_faces;
    const int* ord_lf;    // [K][C]
    int stride;           // shared-memory row length (>= the most faces of a tile)
};

// One block per tile: every face the tile's cells touch is evaluated once in
// this block (face_contrib) into shared memory, rows [3 NQ][stride]; after a
// barrier each cell sums its faces' rows in the reference's order -- for
// each face in increasing original face id the fluctuation, then the flux
// (TransportStep.hpp:464-466, 529-531) -- and applies the stage update.  The
// sums are those of face_kernel + gather_kernel operation for operation,
// without the face-indexed contribution array in HBM; a face between two
// tiles is evaluated by both, each using its own side.
// Dynamic shared memory: 3 NQ stride doubles.
template <class M, class N, int MINB>
__global__ void __launch_bounds__(128, MINB) flux_tile_kernel(MeshDev m, Opts o, TilesDev tl,
                                                        const double* __restrict__ fs,
                                                        const double* __restrict__ aux,
                                                        const double* __restrict__ params, double t_host,
                                                        const double* t_dev, double stage_frac,
                                                        const double* __restrict__ dt_step,
                                                        const int* __restrict__ active, int mode,
                                                        const double* x_in, double* x_out, double* base,
                                                        double* __restrict__ xl_out) {
    constexpr int NQ = M::n_dof_q;
    extern __shared__ double rows[];
    const int b = blockIdx.x;
    const int f0 = tl.face_off[b], nown = tl.face_off[b + 1] - f0;
    const int i0 = tl.in_off[b], nf = nown + tl.in_off[b + 1] - i0;
    const int st = tl.stride;
    for (int lf = threadIdx.x; lf < nf; lf += blockDim.x) {
        const int f = lf < nown ? f0 + lf : tl.in_faces[i0 + lf - nown];
        face_contrib<M, N>(m, f, fs, aux, params, t_host, t_dev, stage_frac, dt_step, active, rows + lf,
                           (size_t)st);
    }
    __syncthreads();
    const int C = m.C, K = m.K;
    const int c1 = tl.cell_off[b + 1];
    for (int c = tl.cell_off[b] + threadIdx.x; c < c1; c += blockDim.x) {
        const int I = cell_instance(m, c);
        if (active && !active[I]) continue;
        double acc[NQ];
#pragma unroll
        for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
        for (int j = 0; j < K; ++j) {
            const int e = tl.ord_lf[j * C + c];
            if (e < 0) continue;
            const double* rw = rows + (e >> 1);
            if (e & 1) {   // the cell is the face's support[0]
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= rw[i * st];
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= rw[(2 * NQ + i) * st];
            } else {
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] -= rw[(NQ + i) * st];
#pragma unroll
                for (int i = 0; i < NQ; ++i) acc[i] += rw[(2 * NQ + i) * st];
            }
        }
        stage_update<M>(m, o, c, I, acc, mode, x_in, x_out, base, dt_step, aux, params, xl_out);
    }
}

}  // namespace zsme
