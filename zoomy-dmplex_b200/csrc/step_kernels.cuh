// Device kernels of the SME step, templated on a generated model plugin
// (Model<T>, Numerics<T>).  All state lives in HBM as one FP64 array per
// variable ("SoA"), cells in Hilbert order.  A solver holds one or several
// independent instances (meshes) concatenated cell- and face-wise; every
// kernel finds a cell's instance in cell_inst (nullptr: one instance) and
// takes that instance's parameters, time, dt and activity.
//
// One SSP stage = prep_kernel + face_kernel + gather_kernel:
//   prep_kernel   per cell: neighbour bounds of the clamped stage state,
//                 gradient of the unclamped one (least squares or Green-Gauss),
//                 limited linear reconstruction at each of the cell's faces ->
//                 face-indexed face states (TransportStep.hpp:196-230, 122-154,
//                 339; Gradient.hpp; Reconstruction.hpp:203-243)
//   face_kernel   per face, once: Riemann flux + fluctuations (face_kernels.cuh)
//   gather_kernel per cell: face contributions in the reference's order, /
//                 volume, SSP-RK(s,2) stage combination, and for the next
//                 stage the state's wet/dry clamp (update_variables) beside
//                 the state itself (face_kernels.cuh)
// After the last stage:
//   finalize_kernel per cell: constraints, implicit Newton source, constraints,
//                 CFL ratio r_c / lambda_c, per-instance minimum (source_kernels.cuh)
//   end_step_kernel per instance: CFL dt, time advance; begin_step_kernel: the
//                 next dt clamped to land on t_end (MUSCLSolver.hpp:141-149)
#pragma once
#include <cfloat>
#include <cstdint>

namespace zsme {

// ------------------------------------------------------------------ layout
struct MeshDev {
    int C;                 // cells (all instances)
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
    const int* face_L;     // [F] support[0]
    const int* face_R;     // [F] support[1] or -1
    const int* face_bc;    // [F] -1 interior, >= 0 bc index, -2 no condition
    const int* cell_inst;  // [C] instance of each cell, or nullptr (one instance)
    const int* face_inst;  // [F] instance of each face, or nullptr
    int np;                // parameters per instance
};

// Per-instance step state ([n_inst] each).
struct StepDev {
    double* t;                 // simulated time
    double* dt_cfl;            // CFL dt of the current state
    double* dt_step;           // dt of the step being taken (clamped to t_end), 0 if inactive
    int* active;               // 1 while t < t_end
    unsigned long long* ratio; // min r_c / lambda_c of the step, as ordered bits of a positive double
    const double* dts;         // imposed dts of a single instance (or nullptr)
    int* step_idx;             // steps taken by instance 0 (index into dts)
    int n_inst;
    double t_end, cfl, dt_max;
    int* diag;                 // [0] nonfinite, [1] negative depth, [2] newton unconverged, [3] MOOD cells,
                               // [6] cells deferred to the generic Newton path (summed over steps)
    int* fallback;             // [C] cells finalize_kernel deferred to finalize_fallback_kernel
    int* n_fallback;           // their count
};

// bits of DBL_MAX: "no cell constrains dt"
#define ZSME_RATIO_NONE 0x7FEFFFFFFFFFFFFFULL

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
__device__ __forceinline__ int cell_instance(const MeshDev& m, int c) { return m.cell_inst ? m.cell_inst[c] : 0; }
__device__ __forceinline__ int face_instance(const MeshDev& m, int f) { return m.face_inst ? m.face_inst[f] : 0; }

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

// The state part of constrain<M> alone: the aux update does not change q.
template <class M>
__device__ __forceinline__ void clamp_q(double* q, const double* a, const double* p) {
    if constexpr (HasUpdateVariables<M>::value) {
        auto r = M::update_variables(q, a, p, 0.0);
#pragma unroll
        for (int i = 0; i < M::n_dof_q; ++i) q[i] = r[i];
    }
}

template <int NQ>
__device__ __forceinline__ void load_q(const double* __restrict__ w, int C, int c, double* q) {
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = w[(size_t)i * C + c];
}

// wl = update_variables(w) for cells [c0, c0 + cn): the clamped copy of a
// state given from outside (zsme_rhs).  Inside a step the gather kernel
// writes it alongside each stage state.
template <class M>
__global__ void __launch_bounds__(128) clamp_kernel(MeshDev m, int c0, int cn, const double* __restrict__ w,
                                                    const double* __restrict__ aux,
                                                    const double* __restrict__ params, double* __restrict__ wl) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r, C = m.C;
    const double* p = params + (size_t)cell_instance(m, c) * m.np;
    double q[NQ], a[NA];
    load_q<NQ>(w, C, c, q);
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    clamp_q<M>(q, a, p);
#pragma unroll
    for (int i = 0; i < NQ; ++i) wl[(size_t)i * C + c] = q[i];
}

// ----------------------------------------------------------------- prep
// The cell's slots in cone order (neighbour, face, side of the face, face
// centroid - cell centroid) and the gradient of the unclamped stage state w:
// least squares in cone order (Gradient.hpp:330-346) or Green-Gauss in
// increasing original face order (Gradient.hpp:91-176), / volume.
template <class M, int KM>
__device__ __forceinline__ void cell_slots_gradient(const MeshDev& m, const Opts& o, int c, int K,
                                                    const double* __restrict__ w, const double* p, int (&nb)[KM],
                                                    int (&ff)[KM], int (&sd)[KM], double (&dx)[KM][M::dimension],
                                                    double (&g)[M::n_dof_q * M::dimension]) {
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    const int C = m.C, F = m.F;
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
    // gradient of the unclamped stage state
#pragma unroll
    for (int i = 0; i < NQ * DIM; ++i) g[i] = 0.0;
    if (o.gradient == 1) {
        // least squares, cone order (Gradient.hpp:330-346)
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (nb[k] < 0) continue;
            const int n = nb[k];
            double wk[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[((size_t)k * 2 + d) * C + c];
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const double du = w[(size_t)i * C + n] - w[(size_t)i * C + c];
#pragma unroll
                for (int d = 0; d < DIM; ++d) g[i * DIM + d] += wk[d] * du;
            }
        }
    } else {
        // Green-Gauss in increasing original face order (Gradient.hpp:91-176)
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
                        const double v = fv * Nf[d];
                        if (isL) g[i * DIM + d] += v;
                        else g[i * DIM + d] -= v;
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
        const double v = m.vol[c];
        if (v > 1e-15) {
#pragma unroll
            for (int i = 0; i < NQ * DIM; ++i) g[i] /= v;
        }
    }
}

// cells [c0, c0 + cn)
// w: the stage state (its gradient), wl: the same state after update_variables
// (bounds and reconstruction base; TransportStep.hpp:326-339 clamp a local
// copy and take the gradient of the unclamped global vector).  The kernel
// works one component at a time and keeps only the gradient and one running
// alpha per face in registers: the components meet only in the limiter's
// alpha = min over components, so a first pass over the components lowers each
// face's alpha and a second writes q + alpha * delta.  Every sum runs in the
// reference's order (cone order for the bounds and least squares, original
// face order for Green-Gauss), so the result is that of the whole-vector form.
// MINB: resident blocks per SM the register allocation must allow (1 = no cap)
// KM: face slots per cell, 3 = exactly three (triangles), 4 = up to four
template <class M, int MINB, int KM>
__global__ void __launch_bounds__(128, MINB) prep_kernel(MeshDev m, Opts o, int c0, int cn, const double* __restrict__ w,
                                                   const double* __restrict__ wl, const double* __restrict__ aux,
                                                   const double* __restrict__ params, double* __restrict__ fs,
                                                   const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, DIM = M::dimension;
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double* p = params + (size_t)I * m.np;
    if (o.order < 2) {
        double ql[NQ], a[NA];
        load_q<NQ>(w, C, c, ql);
#pragma unroll
        for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
        clamp_q<M>(ql, a, p);
        for (int k = 0; k < K; ++k) {
            const int f = m.slot_face[k * C + c];
            if (f < 0) continue;
            const int side = meta_isL(m.slot_meta[k * C + c]) ? 0 : 1;
#pragma unroll
            for (int i = 0; i < NQ; ++i) fs[((size_t)side * NQ + i) * F + f] = ql[i];
        }
        return;
    }
    int nb[KM], ff[KM], sd[KM];
    double dx[KM][DIM], g[NQ * DIM];
    cell_slots_gradient<M, KM>(m, o, c, K, w, p, nb, ff, sd, dx, g);
    // pass 1: each face's alpha = min over components of min(vacuum, tvd)
    // (Reconstruction.hpp:25-36, 62-81, 224-238); "<" ignores NaN as there
    double al[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) al[k] = 1.0;
    if (o.limiter) {
        bool vac = false;
        if (NQ > 1) {   // VacuumLimiter: minimum depth (component 1) over the cell and its neighbours
            double mnh = wl[C + c];
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                if (nb[k] < 0) continue;
                const double v = wl[(size_t)C + nb[k]];
                if (v < mnh) mnh = v;
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
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    if (nb[k] < 0) continue;
                    const double v = wl[(size_t)i * C + nb[k]];
                    if (v < mn) mn = v;
                    if (v > mx) mx = v;
                }
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    if (ff[k] < 0) continue;
                    double d = 0.0;
#pragma unroll
                    for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
                    const double qfu = q + d;
                    const double dq = qfu - q;
                    // TVDLimiter (Reconstruction.hpp:67-78) as selects: the bound on
                    // dq's side, "0" when the cell is that side's extreme.  fmin(1,
                    // r / dq) is exactly 1 when r >= dq > 0 (or r <= dq < 0): the
                    // correctly rounded quotient of |r| >= |dq| is >= 1, so only the
                    // rare limiting case divides (NaN still divides)
                    const bool pos = dq > 0;
                    const double rr = (pos ? mx : mn) - q;
                    const bool room = pos ? (mx > q) : (mn < q);
                    const bool lim = !(pos ? (rr >= dq) : (rr <= dq));
                    const bool small = fabs(dq) < 1e-12;
                    double a = small ? 1.0 : (room ? 1.0 : 0.0);
                    if (!small && room && lim) a = fmin(1.0, rr / dq);
                    if (a < al[k]) al[k] = a;
                }
            }
        }
    }
    // pass 2: face states q + alpha * delta
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double q = wl[(size_t)i * C + c];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (ff[k] < 0) continue;
            double d = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
            fs[((size_t)sd[k] * NQ + i) * F + ff[k]] = q + al[k] * d;
        }
    }
}

// ------------------------------------------------- prep, recording its decisions
// prep_kernel's order-2 face states (positivity "none"), bit for bit, for the
// adjoint's replay: besides the face states it records what the reverse
// sweep needs of the reconstruction, so that adj_cell_kernel need not
// recompute it.  dec [NQ DIM + 3 K][C]: the gradient rows, then per face slot
// k the limiter's alpha, the dq of the branch that set it, and the branch
// (js + 1) + 256 (ks + 1) (js: the component whose ratio set alpha, -1 for a
// 0 / 1 branch; ks: the neighbour slot of that bound, -1 if none), all as
// doubles.  The limiter runs as adj_cell_kernel's replay of it does (the same
// branches, tie rules and first-minimum choice), with the values of
// prep_kernel's selects.
template <class M, int KM>
__global__ void __launch_bounds__(128) prep_tape_kernel(MeshDev m, Opts o, int c0, int cn, const double* __restrict__ w,
                                                        const double* __restrict__ wl,
                                                        const double* __restrict__ params, double* __restrict__ fs,
                                                        double* __restrict__ dec, const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double* p = params + (size_t)I * m.np;
    int nb[KM], ff[KM], sd[KM];
    double dx[KM][DIM], g[NQ * DIM];
    cell_slots_gradient<M, KM>(m, o, c, K, w, p, nb, ff, sd, dx, g);
    double al[KM], dqs[KM];
    int js[KM], ks[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) { al[k] = 1.0; dqs[k] = 1.0; js[k] = -1; ks[k] = -1; }
    if (o.limiter) {
        bool vac = false;
        if (NQ > 1) {
            double mnh = wl[C + c];
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                if (nb[k] < 0) continue;
                const double v = wl[(size_t)C + nb[k]];
                if (v < mnh) mnh = v;
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
                    const double v = wl[(size_t)i * C + nb[k]];
                    if (v < mn) { mn = v; kmn = k; }
                    if (v > mx) { mx = v; kmx = k; }
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
    // face states q + alpha * delta
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double q = wl[(size_t)i * C + c];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (ff[k] < 0) continue;
            double d = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
            fs[((size_t)sd[k] * NQ + i) * F + ff[k]] = q + al[k] * d;
        }
    }
#pragma unroll
    for (int i = 0; i < NQ * DIM; ++i) dec[(size_t)i * C + c] = g[i];
    for (int k = 0; k < K; ++k) {
        dec[((size_t)NQ * DIM + k) * C + c] = al[k];
        dec[((size_t)NQ * DIM + K + k) * C + c] = dqs[k];
        dec[((size_t)NQ * DIM + 2 * K + k) * C + c] = (double)((js[k] + 1) + 256 * (ks[k] + 1));
    }
}

// ---------------------------------------------------------- prep, lean form
// prep_kernel's order-2 face states (positivity "none") with less integer and
// branch work, bit for bit the same:
//  * per-component base pointers and 32-bit element offsets (the host uses
//    this kernel only when 2 NQ F and NQ C fit in an int);
//  * a missing neighbour (boundary slot) is replaced by the cell itself in the
//    limiter bounds and the vacuum minimum, where a comparison with the cell's
//    own value never changes the running minimum or maximum (NaN included);
//  * the Green-Gauss orientation is folded into a signed normal: g - fv N is
//    g + fv (-N) exactly in IEEE arithmetic, and qc + qn equals qn + qc.
// Sums run in the reference's order as in prep_kernel: least squares in cone
// order, Green-Gauss in increasing original face order, bounds in cone order.
template <class M, int MINB, int KM>
__global__ void __launch_bounds__(128, MINB) prep_lean_kernel(MeshDev m, Opts o, int c0, int cn,
                                                        const double* __restrict__ w,
                                                        const double* __restrict__ wl,
                                                        const double* __restrict__ params,
                                                        double* __restrict__ fs, const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double* p = params + (size_t)I * m.np;
    int nbc[KM], fso[KM];
    bool hasn[KM];
    double dx[KM][DIM];
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        int n = -2, f = -1, side = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) dx[k][d] = 0.0;
        if (k < K) {
            n = m.slot_nbr[k * C + c];
            f = m.slot_face[k * C + c];
            side = meta_isL(m.slot_meta[k * C + c]) ? 0 : 1;
#pragma unroll
            for (int d = 0; d < DIM; ++d) dx[k][d] = m.slot_dx[(k * 2 + d) * C + c];
        }
        hasn[k] = n >= 0;
        nbc[k] = n >= 0 ? n : c;
        fso[k] = f >= 0 ? side * NQ * F + f : -1;
    }
    double g[NQ * DIM];
#pragma unroll
    for (int i = 0; i < NQ * DIM; ++i) g[i] = 0.0;
    if (o.gradient == 1) {   // least squares, cone order (Gradient.hpp:330-346)
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (!hasn[k]) continue;
            double wk[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[(k * 2 + d) * C + c];
            const double* wp = w;
#pragma unroll
            for (int i = 0; i < NQ; ++i, wp += C) {
                const double du = wp[nbc[k]] - wp[c];
#pragma unroll
                for (int d = 0; d < DIM; ++d) g[i * DIM + d] += wk[d] * du;
            }
        }
    } else {                 // Green-Gauss, increasing original face order (Gradient.hpp:91-176)
        const int ord = m.order[c];
#pragma unroll
        for (int j = 0; j < KM; ++j) {
            if (j >= K) continue;
            const int k = (ord >> (2 * j)) & 3;
            const int f = m.slot_face[k * C + c];
            if (f < 0) continue;
            const int meta = m.slot_meta[k * C + c];
            const int n = m.slot_nbr[k * C + c];
            const double Nf[2] = {m.fnr[f], m.fnr[F + f]};
            if (n >= 0) {
                double sN[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) sN[d] = meta_isL(meta) ? Nf[d] : -Nf[d];
                const double* wp = w;
#pragma unroll
                for (int i = 0; i < NQ; ++i, wp += C) {
                    const double fv = 0.5 * (wp[c] + wp[n]);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[i * DIM + d] += fv * sN[d];
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
        const double v = m.vol[c];
        if (v > 1e-15) {
#pragma unroll
            for (int i = 0; i < NQ * DIM; ++i) g[i] /= v;
        }
    }
    // pass 1: each face's alpha = min over components of min(vacuum, tvd)
    double al[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) al[k] = 1.0;
    if (o.limiter) {
        bool vac = false;   // VacuumLimiter: minimum depth (component 1) over the cell and its neighbours
        if constexpr (NQ > 1) {
            double mnh = wl[C + c];
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                const double v = wl[C + nbc[k]];
                if (v < mnh) mnh = v;
            }
            vac = mnh < 1e-2;
        }
        if (vac) {
#pragma unroll
            for (int k = 0; k < KM; ++k) al[k] = 0.0;
        } else {
            const double* wp = wl;
#pragma unroll
            for (int i = 0; i < NQ; ++i, wp += C) {
                const double q = wp[c];
                double mn = q, mx = q;
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    const double v = wp[nbc[k]];
                    if (v < mn) mn = v;
                    if (v > mx) mx = v;
                }
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    if (fso[k] < 0) continue;
                    double d = 0.0;
#pragma unroll
                    for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
                    const double qfu = q + d;
                    const double dq = qfu - q;
                    const bool pos = dq > 0;
                    const double rr = (pos ? mx : mn) - q;
                    const bool room = pos ? (mx > q) : (mn < q);
                    const bool lim = !(pos ? (rr >= dq) : (rr <= dq));
                    const bool small = fabs(dq) < 1e-12;
                    double a = small ? 1.0 : (room ? 1.0 : 0.0);
                    if (!small && room && lim) a = fmin(1.0, rr / dq);
                    if (a < al[k]) al[k] = a;
                }
            }
        }
    }
    // pass 2: face states q + alpha * delta
    const double* wp = wl;
#pragma unroll
    for (int i = 0; i < NQ; ++i, wp += C) {
        const double q = wp[c];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (fso[k] < 0) continue;
            double d = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
            fs[fso[k] + i * F] = q + al[k] * d;
        }
    }
}

// ---------------------------------------------------- prep, split over threads
// prep_lean_kernel's face states with P threads per cell: thread part p owns
// components [p NC, p NC + NC), NC = ceil(NQ / P), and keeps only their
// gradient rows in registers, so the kernel needs far fewer registers and runs
// more warps per SM to hide its gathered neighbour loads.  A block holds CB
// cells (a multiple of 32, so each warp serves one part) times P parts; the
// warps of part p load the CB cells' geometry and their components coalesced.
// The limiter's alpha = min over components meets in shared memory: each part
// lowers its own copy of every face's alpha from 1.0 over its components,
// then every part takes the minimum of the P copies.  With the comparisons of
// the one-thread form ("<" skips NaN, and every candidate alpha is in [0, 1]
// or NaN), the minimum of minima is the same value, so the face states are
// bit for bit those of prep_lean_kernel.  The vacuum test reads only the depth
// of the cell and its neighbours and is evaluated by every part alike.
template <int P>
struct SplitShape {
    static constexpr int CB = P == 2 ? 64 : 32;   // cells per block
    static constexpr int threads = CB * P;
};

template <class M, int MINB, int KM, int P>
__global__ void __launch_bounds__(128, MINB) prep_split_kernel(MeshDev m, Opts o, int c0, int cn,
                                                         const double* __restrict__ w,
                                                         const double* __restrict__ wl,
                                                         const double* __restrict__ params,
                                                         double* __restrict__ fs, const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    constexpr int CB = SplitShape<P>::CB, NC = (NQ + P - 1) / P;
    __shared__ double al_sh[P][KM][CB];
    __shared__ double qb_sh[KM][NQ][CB];   // Green-Gauss boundary values of the block's boundary slots
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int part = threadIdx.x / CB, lc = threadIdx.x - part * CB;
    const int r = blockIdx.x * CB + lc;
    const int i0 = part * NC;
    const int c = c0 + r;
    bool live = r < cn;
    int I = 0;
    if (live) {
        I = cell_instance(m, c);
        if (active && !active[I]) live = false;
    }
    if (o.gradient != 1) {
        // the boundary condition of every boundary slot, evaluated once (by the
        // part k mod P) before anything else is held in registers, so that its
        // full-state temporaries do not set the kernel's register count
        if (live) {
            const double* p = params + (size_t)I * m.np;
#pragma unroll
            for (int k = part; k < KM; k += P) {
                if (k >= K) continue;
                const int f = m.slot_face[k * C + c];
                const int meta = m.slot_meta[k * C + c];
                if (f < 0 || m.slot_nbr[k * C + c] >= 0 || meta_bc(meta) < 0) continue;
                double qg[NQ];
                load_q<NQ>(w, C, c, qg);
                const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
                const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
                const auto qb = M::boundary_conditions(meta_bc(meta), qg, (const double*)nullptr, p, nh, xf, 0.0, 0.0);
#pragma unroll
                for (int i = 0; i < NQ; ++i) qb_sh[k][i][lc] = qb[i];
            }
        }
        __syncthreads();
    }
    int nbc[KM], fso[KM];
    bool hasn[KM];
    double dx[KM][DIM], g[NC * DIM], al[KM];
#pragma unroll
    for (int k = 0; k < KM; ++k) al[k] = 1.0;
    if (live) {
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            int n = -2, f = -1, side = 0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) dx[k][d] = 0.0;
            if (k < K) {
                n = m.slot_nbr[k * C + c];
                f = m.slot_face[k * C + c];
                side = meta_isL(m.slot_meta[k * C + c]) ? 0 : 1;
#pragma unroll
                for (int d = 0; d < DIM; ++d) dx[k][d] = m.slot_dx[(k * 2 + d) * C + c];
            }
            hasn[k] = n >= 0;
            nbc[k] = n >= 0 ? n : c;
            fso[k] = f >= 0 ? side * NQ * F + f : -1;
        }
#pragma unroll
        for (int i = 0; i < NC * DIM; ++i) g[i] = 0.0;
        if (o.gradient == 1) {   // least squares, cone order (Gradient.hpp:330-346)
#pragma unroll
            for (int k = 0; k < KM; ++k) {
                if (!hasn[k]) continue;
                double wk[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) wk[d] = m.slot_w[(k * 2 + d) * C + c];
                const double* wp = w + i0 * C;
#pragma unroll
                for (int i = 0; i < NC; ++i, wp += C) {
                    if (i0 + i >= NQ) break;
                    const double du = wp[nbc[k]] - wp[c];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[i * DIM + d] += wk[d] * du;
                }
            }
        } else {                 // Green-Gauss, increasing original face order (Gradient.hpp:91-176)
            const int ord = m.order[c];
#pragma unroll
            for (int j = 0; j < KM; ++j) {
                if (j >= K) continue;
                const int k = (ord >> (2 * j)) & 3;
                const int f = m.slot_face[k * C + c];
                if (f < 0) continue;
                const int meta = m.slot_meta[k * C + c];
                const int n = m.slot_nbr[k * C + c];
                const double Nf[2] = {m.fnr[f], m.fnr[F + f]};
                if (n >= 0) {
                    double sN[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) sN[d] = meta_isL(meta) ? Nf[d] : -Nf[d];
                    const double* wp = w + i0 * C;
#pragma unroll
                    for (int i = 0; i < NC; ++i, wp += C) {
                        if (i0 + i >= NQ) break;
                        const double fv = 0.5 * (wp[c] + wp[n]);
#pragma unroll
                        for (int d = 0; d < DIM; ++d) g[i * DIM + d] += fv * sN[d];
                    }
                } else if (meta_bc(meta) >= 0) {
#pragma unroll
                    for (int i = 0; i < NC; ++i) {
                        if (i0 + i >= NQ) break;
                        const double qb = qb_sh[k][i0 + i][lc];
#pragma unroll
                        for (int d = 0; d < DIM; ++d) g[i * DIM + d] += qb * Nf[d];
                    }
                }
            }
            const double v = m.vol[c];
            if (v > 1e-15) {
#pragma unroll
                for (int i = 0; i < NC * DIM; ++i) g[i] /= v;
            }
        }
        // pass 1: this part's alpha per face = min over its components
        if (o.limiter) {
            bool vac = false;   // VacuumLimiter: minimum depth (component 1) over the cell and its neighbours
            if constexpr (NQ > 1) {
                double mnh = wl[C + c];
#pragma unroll
                for (int k = 0; k < KM; ++k) {
                    const double v = wl[C + nbc[k]];
                    if (v < mnh) mnh = v;
                }
                vac = mnh < 1e-2;
            }
            if (vac) {
#pragma unroll
                for (int k = 0; k < KM; ++k) al[k] = 0.0;
            } else {
                const double* wp = wl + i0 * C;
#pragma unroll
                for (int i = 0; i < NC; ++i, wp += C) {
                    if (i0 + i >= NQ) break;
                    const double q = wp[c];
                    double mn = q, mx = q;
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        const double v = wp[nbc[k]];
                        if (v < mn) mn = v;
                        if (v > mx) mx = v;
                    }
#pragma unroll
                    for (int k = 0; k < KM; ++k) {
                        if (fso[k] < 0) continue;
                        double d = 0.0;
#pragma unroll
                        for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
                        const double qfu = q + d;
                        const double dq = qfu - q;
                        const bool pos = dq > 0;
                        const double rr = (pos ? mx : mn) - q;
                        const bool room = pos ? (mx > q) : (mn < q);
                        const bool lim = !(pos ? (rr >= dq) : (rr <= dq));
                        const bool small = fabs(dq) < 1e-12;
                        double a = small ? 1.0 : (room ? 1.0 : 0.0);
                        if (!small && room && lim) a = fmin(1.0, rr / dq);
                        if (a < al[k]) al[k] = a;
                    }
                }
            }
        }
    }
    if (o.limiter) {   // the parts' minima meet (every thread of the block reaches this barrier)
#pragma unroll
        for (int k = 0; k < KM; ++k) al_sh[part][k][lc] = al[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            double a = 1.0;
#pragma unroll
            for (int q = 0; q < P; ++q) {
                const double v = al_sh[q][k][lc];
                if (v < a) a = v;
            }
            al[k] = a;
        }
    }
    if (!live) return;
    // pass 2: this part's face states q + alpha * delta
    const double* wp = wl + i0 * C;
#pragma unroll
    for (int i = 0; i < NC; ++i, wp += C) {
        if (i0 + i >= NQ) break;
        const double q = wp[c];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (fso[k] < 0) continue;
            double d = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) d += g[i * DIM + e] * dx[k][e];
            fs[fso[k] + (i0 + i) * F] = q + al[k] * d;
        }
    }
}

// Venkatakrishnan eps^2 = vol^(2/dim) (TransportStep.hpp:279), exact in 1-D and 2-D.
template <int DIM>
__host__ __device__ __forceinline__ double venkat_eps2(double v) {
    if constexpr (DIM == 2) return v;
    else if constexpr (DIM == 1) return v * v;
    else return pow(v, 2.0 / DIM);
}

// ---------------------------------------------------- prep, positivity variants
// Order-2 face states of the positivity variants (zhang_shu, mood), cells
// [c0, c0 + cn), layout [b, h, momenta...]:
// 1. the raw gradient of the unclamped stage state w, as prep_kernel;
// 2. TransportStep::LimitGradientsWB (TransportStep.hpp:241-323): per W
//    component (b, eta = b + h, momenta; from the clamped state wl) the
//    Venkatakrishnan factor phi = min over the cell's faces, phi = 0 in dry
//    cells (h < wet_dry_eps), b and momentum factors capped by eta's, the
//    Zhang-Shu theta from the smallest face depth of the depth deviation
//    sh = phi_eta grad eta - phi_b grad b (theta = 1 under MOOD), and the
//    effective gradients phi_b grad b, phi_b grad b + theta sh, theta phi grad m;
// 3. WBPositivityReconstructor::Reconstruct (Reconstruction.hpp:264-286) at
//    each face: b_f, eta_f from the effective gradients, h_f = max(eta_f - b_f, 0),
//    momenta zero where h_f < wet_dry_eps.
// std::min / std::max are written out as the selects they are, so NaN
// propagates as in the reference.  positivity: ZSME_POSITIVITY_ZHANG_SHU or
// _MOOD (no theta); eps: wet_dry_eps.  MINB: the register cap, as prep_kernel's.
template <class M, int KM, int MINB>
__global__ void __launch_bounds__(128, MINB) prep_wb_kernel(MeshDev m, Opts o, int positivity, double eps, int c0, int cn,
                                                      const double* __restrict__ w, const double* __restrict__ wl,
                                                      const double* __restrict__ params, double* __restrict__ fs,
                                                      const int* __restrict__ active) {
    constexpr int NQ = M::n_dof_q, DIM = M::dimension;
    constexpr int B = 0, H = 1;
    const int C = m.C, F = m.F;
    const int K = KM == 3 ? 3 : m.K;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int I = cell_instance(m, c);
    if (active && !active[I]) return;
    const double* p = params + (size_t)I * m.np;
    int nb[KM], ff[KM], sd[KM];
    double dx[KM][DIM], g[NQ * DIM];
    cell_slots_gradient<M, KM>(m, o, c, K, w, p, nb, ff, sd, dx, g);
    double geta[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) geta[d] = g[H * DIM + d] + g[B * DIM + d];
    const double h_bar = wl[(size_t)H * C + c], b_bar = wl[(size_t)B * C + c];
    const double eps2 = venkat_eps2<DIM>(m.vol[c]);
    double phi[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const double wc = i == H ? (b_bar + h_bar) : wl[(size_t)i * C + c];
        double wmn = wc, wmx = wc;
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (nb[k] < 0) continue;
            const int n = nb[k];
            const double wn = i == H ? (wl[(size_t)B * C + n] + wl[(size_t)H * C + n]) : wl[(size_t)i * C + n];
            if (wn < wmn) wmn = wn;
            if (wn > wmx) wmx = wn;
        }
        double ph = 1.0;
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (ff[k] < 0) continue;
            double delta = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) delta += (i == H ? geta[d] : g[i * DIM + d]) * dx[k][d];
            if (fabs(delta) < 1e-14) continue;
            const double dm = (delta > 0) ? (wmx - wc) : (wmn - wc);
            const double num = dm * dm + eps2 + 2 * delta * dm;
            const double den = dm * dm + 2 * delta * delta + delta * dm + eps2;
            double pf = (den > 1e-30) ? num / den : 1.0;
            pf = (pf < 1.0) ? pf : 1.0;   // std::min(1, pf)
            pf = (0.0 < pf) ? pf : 0.0;   // std::max(0, pf)
            if (pf < ph) ph = pf;
        }
        phi[i] = ph;
    }
    if (h_bar < eps) {
#pragma unroll
        for (int i = 0; i < NQ; ++i) phi[i] = 0.0;
    }
    phi[B] = (phi[H] < phi[B]) ? phi[H] : phi[B];
#pragma unroll
    for (int i = 0; i < NQ; ++i)
        if (i != B && i != H) phi[i] = (phi[H] < phi[i]) ? phi[H] : phi[i];
    double sh[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) sh[d] = phi[H] * geta[d] - phi[B] * g[B * DIM + d];
    double hmin = h_bar;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        if (ff[k] < 0) continue;
        double hf = h_bar;
#pragma unroll
        for (int d = 0; d < DIM; ++d) hf += sh[d] * dx[k][d];
        if (hf < hmin) hmin = hf;
    }
    double theta = 1.0;
    if (positivity != ZSME_POSITIVITY_MOOD && hmin < 0.0) {
        const double gap = h_bar - hmin;
        double th = h_bar / ((gap < 1e-14) ? 1e-14 : gap);
        th = (th < 1.0) ? th : 1.0;
        theta = (0.0 < th) ? th : 0.0;
    }
    // effective gradients in place: b slot grad b_eff, h slot grad eta_eff
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const double gb = g[B * DIM + d];
        g[B * DIM + d] = phi[B] * gb;
        g[H * DIM + d] = phi[B] * gb + theta * sh[d];
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i)
        if (i != B && i != H)
#pragma unroll
            for (int d = 0; d < DIM; ++d) g[i * DIM + d] = theta * phi[i] * g[i * DIM + d];
    // face states
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        if (ff[k] < 0) continue;
        double* out = fs + (size_t)sd[k] * NQ * F + ff[k];
        double db = 0.0, de = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) db += g[B * DIM + d] * dx[k][d];
#pragma unroll
        for (int d = 0; d < DIM; ++d) de += g[H * DIM + d] * dx[k][d];
        const double b_f = b_bar + db;
        const double eta_f = (b_bar + h_bar) + de;
        const double hd = eta_f - b_f;
        const double h_f = (hd < 0.0) ? 0.0 : hd;
        out[(size_t)B * F] = b_f;
        out[(size_t)H * F] = h_f;
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            if (i == B || i == H) continue;
            double di = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) di += g[i * DIM + d] * dx[k][d];
            out[(size_t)i * F] = (h_f < eps) ? 0.0 : (wl[(size_t)i * C + c] + di);
        }
    }
}

// ------------------------------------------------------- derivative aux
// The derivative aux slots a plugin fills through its field-level
// update_aux_variables (one entry per compute_derivative call it makes).
struct DerivSpecs {
    int n;
    int aux[8], comp[8], axis[8], order[8];   // slot, state variable, axis, total derivative order
};

// TransportStep::RefreshDerivativeAux with compute_derivative
// (TransportStep.hpp:161-192, UserFunctions.H:60-112) for cells [c0, c0 + cn):
// per requested slot, the Green-Gauss gradient of state variable comp of x --
// the cell's faces in increasing original face id (the reference's face loop
// order), 0.5 (s_support0 + s_support1) N added when the cell is support[0]
// and subtracted otherwise, s_cell N on every exterior face (zero Neumann) --
// along `axis`, / volume where positive (else 0); order 0 copies the variable.
template <class M>
__global__ void __launch_bounds__(128) derivative_aux_kernel(MeshDev m, DerivSpecs ds, int c0, int cn,
                                                             const double* __restrict__ x,
                                                             double* __restrict__ aux,
                                                             const int* __restrict__ active) {
    constexpr int DIM = M::dimension;
    const int C = m.C, F = m.F;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    if (active && !active[cell_instance(m, c)]) return;
    const int ord = m.order[c];
    for (int e = 0; e < ds.n; ++e) {
        const double* s = x + (size_t)ds.comp[e] * C;
        double result = 0.0;
        if (ds.order[e] == 0) {
            result = s[c];
        } else {
            double g[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) g[d] = 0.0;
            for (int j = 0; j < m.K; ++j) {
                const int k = (ord >> (2 * j)) & 3;
                const int f = m.slot_face[k * C + c];
                if (f < 0) continue;
                const int n = m.slot_nbr[k * C + c];
                const double Nf[2] = {m.fnr[f], m.fnr[F + f]};
                if (n >= 0) {
                    const bool isL = meta_isL(m.slot_meta[k * C + c]);
                    const double fv = 0.5 * (isL ? (s[c] + s[n]) : (s[n] + s[c]));
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        const double v = fv * Nf[d];
                        if (isL) g[d] += v;
                        else g[d] -= v;
                    }
                } else {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[d] += s[c] * Nf[d];
                }
            }
            const double v = m.vol[c];
            if (ds.axis[e] < DIM && v > 0) {
#pragma unroll
                for (int d = 0; d < DIM; ++d)
                    if (d == ds.axis[e]) result = g[d] / v;
            }
        }
        aux[(size_t)ds.aux[e] * C + c] = result;
    }
}

// ------------------------------------------------------------------ MOOD
// Local MOOD (MUSCLSolver.hpp:150-170, 197-229; TransportStep.hpp:363-381,
// 412-418): a cell whose depth after the transport step is below -1e-10 is
// overwritten by its first-order forward-Euler update from the step's start
// state xs -- piecewise-constant clamped states on every face of the cell,
// the face contributions summed in increasing original face order, / volume
// -- and counted in diag[3].  No other cell changes, so each troubled cell
// evaluates its own faces and no face pass is needed.  mood_detect_kernel
// lists the troubled cells of [c0, c0 + cn) (warp-aggregated, so a light
// kernel scans the mesh) and mood_kernel overrides the listed ones; both run
// between the last stage and finalize, whose constraints follow the
// override as EnforcePhysicalConstraints does.
static __global__ void __launch_bounds__(128) mood_detect_kernel(MeshDev m, int c0, int cn, const double* __restrict__ x,
                                                          StepDev sd, int* __restrict__ list, int* __restrict__ count) {
    const int C = m.C;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = c0 + r;
    bool bad = false;
    if (r < cn) {
        const int I = cell_instance(m, c);
        bad = (!sd.active || sd.active[I]) && x[C + c] < -1.0e-10;
    }
    const unsigned bm = __ballot_sync(0xffffffffu, bad);
    if (!bm) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) {
        base = atomicAdd(count, __popc(bm));
        atomicAdd(&sd.diag[3], __popc(bm));
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    if (bad) list[base + __popc(bm & ((1u << lane) - 1u))] = c;
}

template <class M, class N>
__device__ __forceinline__ void mood_cell(const MeshDev& m, int c, double* __restrict__ x,
                                          const double* __restrict__ xs, const double* __restrict__ aux,
                                          const double* __restrict__ params, const StepDev& sd) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int C = m.C, F = m.F;
    const int I = cell_instance(m, c);
    const double* p = params + (size_t)I * m.np;
    const double t = sd.t[I], h = sd.dt_step[I];
    double qc[NQ], ac[NA];
    load_q<NQ>(xs, C, c, qc);
#pragma unroll
    for (int i = 0; i < NA; ++i) ac[i] = aux[(size_t)i * C + c];
    clamp_q<M>(qc, ac, p);
    double acc[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) acc[i] = 0.0;
    const int ord = m.order[c];
    for (int j = 0; j < m.K; ++j) {
        const int k = (ord >> (2 * j)) & 3;
        const int f = m.slot_face[k * C + c];
        if (f < 0) continue;
        const int meta = m.slot_meta[k * C + c];
        const int n = m.slot_nbr[k * C + c];
        if (n < 0 && meta_bc(meta) < 0) continue;
        const double area = m.farea[f];
        const double nh[3] = {m.fn[f], m.fn[F + f], 0.0};
        const double xf[3] = {m.fc[f], m.fc[F + f], 0.0};
        if (n >= 0) {
            double qn[NQ], an[NA];
            load_q<NQ>(xs, C, n, qn);
#pragma unroll
            for (int i = 0; i < NA; ++i) an[i] = aux[(size_t)i * C + n];
            clamp_q<M>(qn, an, p);
            const bool isL = meta_isL(meta);
            const double* qL = isL ? qc : qn;
            const double* qR = isL ? qn : qc;
            double aL[NA], aR[NA];
            {
                auto ra = M::update_aux_variables(qL, isL ? ac : an, p, 0.0, xf);
                auto rb = M::update_aux_variables(qR, isL ? an : ac, p, 0.0, xf);
#pragma unroll
                for (int i = 0; i < NA; ++i) { aL[i] = ra[i]; aR[i] = rb[i]; }
            }
            const auto flux = N::numerical_flux(qL, qR, aL, aR, p, nh);
            const auto nc = N::numerical_fluctuations(qL, qR, aL, aR, p, nh);
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
            {
                auto ra = M::update_aux_variables(qc, ac, p, t, xf);
#pragma unroll
                for (int i = 0; i < NA; ++i) aL[i] = ra[i];
            }
            const auto qR = M::boundary_conditions(meta_bc(meta), qc, aL, p, nh, xf, t, 0.0);
            {
                auto rb = M::update_aux_variables(qR.data, aL, p, t, xf);
#pragma unroll
                for (int i = 0; i < NA; ++i) aR[i] = rb[i];
            }
            const auto flux = N::numerical_flux(qc, qR.data, aL, aR, p, nh);
            const auto nc = N::numerical_fluctuations(qc, qR.data, aL, aR, p, nh);
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
#pragma unroll
    for (int i = 0; i < NQ; ++i) x[(size_t)i * C + c] = xs[(size_t)i * C + c] + h * acc[i];
}

template <class M, class N>
__global__ void __launch_bounds__(64) mood_kernel(MeshDev m, double* __restrict__ x, const double* __restrict__ xs,
                                                  const double* __restrict__ aux, const double* __restrict__ params,
                                                  StepDev sd, const int* __restrict__ list,
                                                  const int* __restrict__ count) {
    const int n = *count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        mood_cell<M, N>(m, list[e], x, xs, aux, params, sd);
}

// --------------------------------------------------------------- step ends
// begin: each instance's dt for this step from its CFL dt (or the imposed
// one), clamped to land on t_end; inactive once t >= t_end.
static __global__ void begin_step_kernel(StepDev sd, int i0, int ni) {
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= i0 + ni) return;
    const double t0 = sd.t[i];
    double d0 = sd.dts ? sd.dts[*sd.step_idx] : sd.dt_cfl[i];
    const int act = t0 < sd.t_end;
    if (t0 + d0 > sd.t_end) d0 = sd.t_end - t0;
    sd.active[i] = act;
    sd.dt_step[i] = act ? d0 : 0.0;
}

// end: the instance's minimum ratio -> CFL dt (or dt_max when no cell
// constrains it, VirtualSolver.hpp:354-356); time advance.  mode 1: step end,
// mode 0: initial dt = max(dt, min_dt) (MUSCLSolver.hpp:103), mode 2: dt
// into dt_out only (ComputeTimeStep without side effects).
static __global__ void end_step_kernel(StepDev sd, int i0, int ni, int mode, double min_dt, double* dt_out) {
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= i0 + ni) return;
    const double r = __longlong_as_double((long long)sd.ratio[i]);
    sd.ratio[i] = ZSME_RATIO_NONE;
    const double dt = (!isfinite(r) || r >= 0.5 * DBL_MAX) ? sd.dt_max : sd.cfl * r;
    if (mode == 1) {
        if (sd.active[i]) {
            sd.t[i] = sd.t[i] + sd.dt_step[i];
            if (i == 0) *sd.step_idx += 1;
            sd.dt_cfl[i] = dt;
        }
    } else if (mode == 0) {
        sd.dt_cfl[i] = dt > min_dt ? dt : min_dt;
    } else {
        dt_out[i] = dt;
    }
}

// ------------------------------------------------------- layout transforms
// AoS (caller order within an instance) <-> SoA (Hilbert order): cells
// [c0, c0 + cn) of the SoA arrays (row stride C) are instance-local rows
// old_of_new[c] of the AoS buffer.
static __global__ void set_time_kernel(double* t, double v) { *t = v; }
// q_aos[e] = state of caller cell cells[e] (ids outside [0, C) are skipped)
static __global__ void get_cells_kernel(const double* __restrict__ soa, int C, int nq,
                                        const int* __restrict__ new_of_old, const int* __restrict__ cells, int n,
                                        double* __restrict__ q_aos) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int o = cells[e];
    if (o < 0 || o >= C) return;
    const int c = new_of_old[o];
    for (int i = 0; i < nq; ++i) q_aos[(size_t)e * nq + i] = soa[(size_t)i * C + c];
}
// the state of caller cell cells[e] = q_aos[e], and its aux recomputed
template <class M>
__global__ void set_cells_kernel(double* __restrict__ x, double* __restrict__ aux, int C,
                                 const int* __restrict__ new_of_old, const int* __restrict__ cells, int n,
                                 const double* __restrict__ q_aos, const double* __restrict__ params) {
    constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int o = cells[e];
    if (o < 0 || o >= C) return;
    const int c = new_of_old[o];
    double q[NQ], a[NA];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        q[i] = q_aos[(size_t)e * NQ + i];
        x[(size_t)i * C + c] = q[i];
    }
#pragma unroll
    for (int i = 0; i < NA; ++i) a[i] = aux[(size_t)i * C + c];
    const double X0[3] = {0.0, 0.0, 0.0};
    const auto ra = M::update_aux_variables(q, a, params, 0.0, X0);
#pragma unroll
    for (int i = 0; i < NA; ++i) aux[(size_t)i * C + c] = ra[i];
}
static __global__ void aos_to_soa_kernel(const double* __restrict__ aos, double* __restrict__ soa,
                                         const int* __restrict__ old_of_new, int c0, int cn, int C, int nq) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int o = old_of_new[c];
    for (int i = 0; i < nq; ++i) soa[(size_t)i * C + c] = aos[(size_t)o * nq + i];
}
static __global__ void soa_to_aos_kernel(const double* __restrict__ soa, double* __restrict__ aos,
                                         const int* __restrict__ old_of_new, int c0, int cn, int C, int nq) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cn) return;
    const int c = c0 + r;
    const int o = old_of_new[c];
    for (int i = 0; i < nq; ++i) aos[(size_t)o * nq + i] = soa[(size_t)i * C + c];
}

}  // namespace zsme
