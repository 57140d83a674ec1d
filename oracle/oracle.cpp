// ORACLE -- test infrastructure, not the product.
//
// A PETSc-free CPU restatement of the reference's SME time step, used only by
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
// checker.  Every routine follows one reference function (cited inline):
//
//   FormRHS            TransportStep.hpp:325-357
//   UpdateState        TransportStep.hpp:196-230
//   UpdateNeighborBounds TransportStep.hpp:122-154 (SetupTopology 106-120)
//   ComputeFluxes      TransportStep.hpp:383-565
//   LeastSquares       Gradient.hpp:196-360 (Setup 222-298, Compute 300-359)
//   GreenGauss         Gradient.hpp:43-191 (BC callback ModularSolver.hpp:68-71)
//   Linear/PCM + Vacuum + TVD  Reconstruction.hpp:23-81, 143-244
//   SourceStep         SourceStep.hpp:26-242
//   ComputeTimeStep    VirtualSolver.hpp:285-357
//   SSP-RK(s,2)        PETSc TSSSP "rks2" (SolverStrategies.hpp:33-35)
//   Euler (order 1)    PETSc TSEULER (SolverStrategies.hpp:37)
//   step loop          MUSCLSolver.hpp:140-188, EnforcePhysicalConstraints 234-254
//
// The face loop computes each face's contributions independently and every
// cell then sums them in increasing face order -- the order in which the
// reference's sequential face loop accumulates -- so the result does not
// depend on the number of OpenMP threads.
//
// Parity status: the pointwise model arithmetic is pinned against the
// reference's own shipped Model.H/Numerics.H compiled here (oracle/_ref); the
// step composition cannot be run from the reference (PETSc is absent) and is
// pinned only by this restatement.
#include "model_prelude.h"
#include "dual.h"
#include "flopcount.h"
#include "zsme.h"

#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>

#include "imex_tableau.h"
#include <vector>

namespace sme1d_l0_malpasset {
#include "sme1d_l0_malpasset/Model.H"
#include "sme1d_l0_malpasset/Numerics.H"
}
namespace sme2d_l0 {
#include "sme2d_l0/Model.H"
#include "sme2d_l0/Numerics.H"
}
namespace sme2d_l1 {
#include "sme2d_l1/Model.H"
#include "sme2d_l1/Numerics.H"
}
namespace sme2d_l2 {
#include "sme2d_l2/Model.H"
#include "sme2d_l2/Numerics.H"
}
namespace sme2d_l4 {
#include "sme2d_l4/Model.H"
#include "sme2d_l4/Numerics.H"
}
#ifdef ORACLE_WITH_REFERENCE_MODEL
// The reference's own generated 1-D level-0 headers (oracle/_ref build only).
// Its field-level update_aux_variables calls compute_derivative on the mesh
// handle of model_prelude.h, which the oracle serves with its restatement of
// the reference's Green-Gauss derivative (Oracle::compute_derivative_gg).
namespace ref1d {
#include "Model.H"
#include "Numerics.H"
}
#endif

namespace {

// Static-chunked parallel loop over [0, n) on std::thread workers.  Each
// index is handled by exactly one worker and no loop here has cross-index
// dependencies, so results do not depend on the thread count.
int g_threads = 1;
template <class Fn>
void par_for(int n, Fn fn) {
    int nt = std::max(1, std::min(g_threads, n / 256 + 1));
    if (nt == 1) {
        for (int i = 0; i < n; ++i) fn(i, 0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([=, &fn] {
            int a = (int)((long long)n * t / nt), b = (int)((long long)n * (t + 1) / nt);
            for (int i = a; i < b; ++i) fn(i, t);
        });
    for (auto& x : th) x.join();
}
int par_width(int n) { return std::max(1, std::min(g_threads, n / 256 + 1)); }

thread_local std::string g_err;
int fail(int code, const std::string& m) {
    g_err = m;
    return code;
}

struct OracleBase {
    virtual ~OracleBase() = default;
    virtual int nq() const = 0;
    virtual int naux() const = 0;
    virtual void set_state(const double* q, double t) = 0;
    virtual void get_state(double* q) const = 0;
    virtual void get_aux(double* a) const = 0;
    virtual void rhs(double t, const double* x, double* f) = 0;
    virtual void update_state() = 0;
    virtual void source(double dt) = 0;
    virtual double compute_dt() = 0;
    virtual void step(int n, const double* dts) = 0;
    virtual void get_time(double* t, double* dt) const = 0;
    virtual void set_params(const double* p) = 0;
    virtual int newton_unconverged() const = 0;
    virtual long long mood_cells() const = 0;
    virtual void gradient(const double* x, double* g) = 0;
    // tangent-linear (dual-number) instances only: seed / read directions
    virtual void set_tangent(const double*, const double*) {}
    virtual void get_tangent(double*) const {}
    // the fully implicit strategy (double instances only)
    virtual void implicit_function(double, const double*, const double*, double*) {}
    virtual void implicit_jacobian(double, const double*, double, double*, double*) {}
    virtual int implicit_stats(int*) const { return 0; }
};

// S: the scalar of state and parameters -- double, Dual<1> for the
// tangent-linear run (derivative along one seeded direction, the branches
// decided by the values exactly as in the double run), or Counted to count
// the step's floating-point operations (flopcount.h).
template <template <typename> class MT, template <typename> class NT, class Scalar = double>
struct Oracle : OracleBase {
    using T = Scalar;
    using M = MT<T>;
    using N = NT<T>;
    static constexpr int NQ = M::n_dof_q;
    static constexpr int NA = M::n_dof_qaux;
    static constexpr int DIM = M::dimension;

    // mesh, caller order
    int C = 0, F = 0, K = 0;
    std::vector<double> cc, vol, fc, fn;
    std::vector<int> cf, fcell, fbc;
    std::vector<int> nb_off, nb_list;    // face neighbours, cone order
    std::vector<double> lsq_w;           // DIM weights per neighbour entry
    std::vector<int> cell_face_sorted;   // each cell's faces, increasing id
    zsme_settings st{};
    std::vector<T> params;
    std::vector<T> X, A, G;
    double time = 0.0, dt = 0.0;
    int n_unconv = 0;
    long long n_troubled = 0;   // cells redone at first order by MOOD, all steps
    std::vector<unsigned char> cfl_skip;   // cells left out of the CFL minimum

    Oracle(const zsme_mesh* m, const zsme_settings* s, const double* p) {
        C = m->n_cells; F = m->n_faces; K = m->max_faces;
        cc.assign(m->cell_centroid, m->cell_centroid + 2 * C);
        vol.assign(m->cell_volume, m->cell_volume + C);
        fc.assign(m->face_centroid, m->face_centroid + 2 * F);
        fn.assign(m->face_normal, m->face_normal + 2 * F);
        cf.assign(m->cell_faces, m->cell_faces + K * C);
        fcell.assign(m->face_cells, m->face_cells + 2 * F);
        fbc.assign(m->face_bc, m->face_bc + F);
        if (m->cell_cfl_skip) cfl_skip.assign(m->cell_cfl_skip, m->cell_cfl_skip + C);
        st = *s;
        // Zhang-Shu positivity holds for CFL <= 1/6 at order 2 (MUSCLSolver.hpp:33-38)
        if (st.reconstruction_order >= 2 && st.positivity == ZSME_POSITIVITY_ZHANG_SHU && st.cfl > 1.0 / 6.0)
            st.cfl = 1.0 / 6.0;
        auto dp = M::default_parameters();
        params.assign(dp.begin(), dp.end());
        if (p) params.assign(p, p + M::n_parameters);
        X.assign((size_t)C * NQ, 0.0);
        A.assign((size_t)C * NA, 0.0);
        G.assign((size_t)C * NQ * DIM, 0.0);
        setup_topology();
        setup_lsq();
    }

    int nq() const override { return NQ; }
    int naux() const override { return NA; }
    // the phase the operation counters of a Counted instance charge
    static void ph(int p) {
        if constexpr (std::is_same<T, zsme::Counted>::value) zsme_flops::phase = p;
    }
    void set_params(const double* p) override { params.assign(p, p + M::n_parameters); }
    int newton_unconverged() const override { return n_unconv; }
    long long mood_cells() const override { return n_troubled; }

    // SetupTopology (TransportStep.hpp:106-120): adjacency of a cell = the
    // other cells of its faces in cone order.
    void setup_topology() {
        nb_off.assign(C + 1, 0);
        nb_list.clear();
        cell_face_sorted.assign((size_t)C * K, -1);
        for (int c = 0; c < C; ++c) {
            std::vector<int> fs;
            for (int k = 0; k < K; ++k) {
                int f = cf[(size_t)c * K + k];
                if (f < 0) continue;
                fs.push_back(f);
                int a = fcell[2 * f], b = fcell[2 * f + 1];
                int o = (a == c) ? b : a;
                if (o < 0 || o == c) continue;
                bool dup = false;
                for (int q = nb_off[c]; q < (int)nb_list.size(); ++q) dup |= nb_list[q] == o;
                if (!dup) nb_list.push_back(o);
            }
            std::sort(fs.begin(), fs.end());
            for (size_t k = 0; k < fs.size(); ++k) cell_face_sorted[(size_t)c * K + k] = fs[k];
            nb_off[c + 1] = (int)nb_list.size();
        }
    }

    // LeastSquaresGradient::Setup (Gradient.hpp:222-298), order 1 basis.
    static bool solve_spd(int n, std::vector<double>& a, std::vector<double>& b) {
        std::vector<double> L(n * n, 0.0);
        for (int i = 0; i < n; i++) {
            for (int j = 0; j <= i; j++) {
                double sum = 0;
                for (int k = 0; k < j; k++) sum += L[i * n + k] * L[j * n + k];
                if (i == j) {
                    double val = a[i * n + i] - sum;
                    if (val <= 0) return false;
                    L[i * n + j] = std::sqrt(val);
                } else {
                    L[i * n + j] = (a[i * n + j] - sum) / L[j * n + j];
                }
            }
        }
        for (int i = 0; i < n; i++) {
            double sum = 0;
            for (int k = 0; k < i; k++) sum += L[i * n + k] * b[k];
            b[i] = (b[i] - sum) / L[i * n + i];
        }
        for (int i = n - 1; i >= 0; i--) {
            double sum = 0;
            for (int k = i + 1; k < n; k++) sum += L[k * n + i] * b[k];
            b[i] = (b[i] - sum) / L[i * n + i];
        }
        return true;
    }

    void setup_lsq() {
        lsq_w.assign(nb_list.size() * DIM, 0.0);
        for (int c = 0; c < C; ++c) {
            std::vector<std::vector<double>> basis;
            for (int q = nb_off[c]; q < nb_off[c + 1]; ++q) {
                int n = nb_list[q];
                std::vector<double> b;
                for (int d = 0; d < DIM; ++d) b.push_back(cc[2 * n + d] - cc[2 * c + d]);
                basis.push_back(b);
            }
            std::vector<double> ata(DIM * DIM, 0.0);
            for (auto& b : basis)
                for (int i = 0; i < DIM; ++i)
                    for (int j = 0; j < DIM; ++j) ata[i * DIM + j] += b[i] * b[j];
            for (size_t k = 0; k < basis.size(); ++k) {
                std::vector<double> rhs = basis[k], sys = ata;
                bool ok = solve_spd(DIM, sys, rhs);
                for (int d = 0; d < DIM; ++d)
                    lsq_w[(size_t)(nb_off[c] + k) * DIM + d] = ok ? rhs[d] : 0.0;
            }
        }
    }

    // ---------------------------------------------------------------- state
    void constrain_cell(T* q, T* a) const {
        if constexpr (zsme::HasUpdateVariables<M>::value) {
            auto r = M::update_variables(q, a, params.data(), 0.0);
            for (int i = 0; i < NQ; ++i) q[i] = r[i];
        }
        const T X0[3] = {0, 0, 0};
        auto ra = M::update_aux_variables(q, a, params.data(), 0.0, X0);
        for (int i = 0; i < NA; ++i) a[i] = ra[i];
    }
    // TransportStep::UpdateState (TransportStep.hpp:196-230): the derivative
    // aux first (when refreshed), then the pointwise clamp and aux per cell.
    void update_state_vec(std::vector<T>& x, std::vector<T>& a) const {
        if (st.refresh_derivative_aux) refresh_derivative_aux(x, a);
        par_for(C, [&](int c, int) { constrain_cell(&x[(size_t)c * NQ], &a[(size_t)c * NA]); });
    }
    // TransportStep::RefreshDerivativeAux (TransportStep.hpp:161-192): the state
    // and aux de-interleaved into per-variable fields, the plugin's field-level
    // update_aux_variables called on them (it fills its derivative slots through
    // compute_derivative), the aux interleaved back.  Plugins without that
    // overload have nothing to refresh; so do the dual-number and counting
    // instances, whose derivative slots feed no state update.
    void refresh_derivative_aux(const std::vector<T>& x, std::vector<T>& a) const {
        if constexpr (zsme::HasFieldAuxUpdate<M>::value && std::is_same<T, double>::value) {
            std::vector<std::vector<double>> Qf(NQ, std::vector<double>(C)), Af(NA, std::vector<double>(C));
            for (int c = 0; c < C; ++c) {
                for (int i = 0; i < NQ; ++i) Qf[i][c] = x[(size_t)c * NQ + i];
                for (int k = 0; k < NA; ++k) Af[k][c] = a[(size_t)c * NA + k];
            }
            std::vector<double*> Qp(NQ), Ap(NA);
            for (int i = 0; i < NQ; ++i) Qp[i] = Qf[i].data();
            for (int k = 0; k < NA; ++k) Ap[k] = Af[k].data();
            const ZoomyMesh mesh{&Oracle::derivative_request, (void*)this};
            M::update_aux_variables(Qp.data(), Ap.data(), 0.0, mesh);
            for (int c = 0; c < C; ++c)
                for (int k = 0; k < NA; ++k) a[(size_t)c * NA + k] = Af[k][c];
        }
    }
    static void derivative_request(const ZoomyMesh& mesh, double* result, const double* source, int dx, int dy,
                                   int dz) {
        static_cast<const Oracle*>(mesh.ctx)->compute_derivative_gg(result, source, dx, dy, dz);
    }
    // compute_derivative (UserFunctions.H:60-112): the Green-Gauss cell gradient
    // of one field -- every face in increasing face order adds 0.5 (s_L + s_R) N
    // to its first cell and subtracts it from its second; a boundary face adds
    // s_cell N (zero Neumann) -- then the requested axis / volume where the
    // volume is positive (0 elsewhere); the identity for order 0.
    void compute_derivative_gg(double* result, const double* src, int dx, int dy, int dz) const {
        const int total = dx + dy + dz;
        const int axis = dx == 1 ? 0 : (dy == 1 ? 1 : 2);
        for (int c = 0; c < C; ++c) result[c] = 0.0;
        if (total == 0) {
            for (int c = 0; c < C; ++c) result[c] = src[c];
            return;
        }
        std::vector<double> grad((size_t)C * DIM, 0.0);
        for (int f = 0; f < F; ++f) {
            const int a = fcell[2 * f], b = fcell[2 * f + 1];
            if (b >= 0) {
                const double fv = 0.5 * (src[a] + src[b]);
                for (int d = 0; d < DIM; ++d) {
                    const double v = fv * fn[2 * f + d];
                    grad[(size_t)a * DIM + d] += v;
                    grad[(size_t)b * DIM + d] -= v;
                }
            } else {
                const double fv = src[a];
                for (int d = 0; d < DIM; ++d) grad[(size_t)a * DIM + d] += fv * fn[2 * f + d];
            }
        }
        if (axis >= DIM) return;
        for (int c = 0; c < C; ++c)
            if (vol[c] > 0) result[c] = grad[(size_t)c * DIM + axis] / vol[c];
    }

    // ------------------------------------------------------------ gradients
    void gradient_lsq(const std::vector<T>& x, std::vector<T>& g) const {
par_for(C, [&](int c, int) {
            T* gc = &g[(size_t)c * NQ * DIM];
            for (int k = 0; k < NQ * DIM; ++k) gc[k] = 0.0;
            const T* qc = &x[(size_t)c * NQ];
            for (int q = nb_off[c]; q < nb_off[c + 1]; ++q) {
                const T* qn = &x[(size_t)nb_list[q] * NQ];
                const double* w = &lsq_w[(size_t)q * DIM];
                for (int i = 0; i < NQ; ++i) {
                    T du = qn[i] - qc[i];
                    for (int d = 0; d < DIM; ++d) gc[i * DIM + d] += w[d] * du;
                }
            }
        });
    }
    // GreenGaussGradient::Compute: face loop, boundary ghost value q_bc * N,
    // then / volume.  Accumulated per cell in increasing face order.
    void gradient_gg(const std::vector<T>& x, std::vector<T>& g) const {
par_for(C, [&](int c, int) {
            T* gc = &g[(size_t)c * NQ * DIM];
            for (int k = 0; k < NQ * DIM; ++k) gc[k] = 0.0;
            for (int k = 0; k < K; ++k) {
                int f = cell_face_sorted[(size_t)c * K + k];
                if (f < 0) break;
                int L = fcell[2 * f], R = fcell[2 * f + 1];
                const double* Nf = &fn[2 * f];
                if (R >= 0) {
                    const T* qL = &x[(size_t)L * NQ];
                    const T* qR = &x[(size_t)R * NQ];
                    for (int i = 0; i < NQ; ++i) {
                        T fv = 0.5 * (qL[i] + qR[i]);
                        for (int d = 0; d < DIM; ++d) {
                            T v = fv * Nf[d];
                            if (c == L) gc[i * DIM + d] += v; else gc[i * DIM + d] -= v;
                        }
                    }
                } else if (fbc[f] >= 0) {
                    T area = 0;
                    for (int d = 0; d < DIM; ++d) area += Nf[d] * Nf[d];
                    area = std::sqrt(area);
                    T nh[3] = {0, 0, 0};
                    for (int d = 0; d < DIM; ++d) nh[d] = Nf[d] / area;
                    const T xf[3] = {fc[2 * f], fc[2 * f + 1], 0.0};
                    auto qb = M::boundary_conditions(fbc[f], &x[(size_t)c * NQ], nullptr, params.data(), nh, xf,
                                                     0.0, 0.0);
                    for (int i = 0; i < NQ; ++i)
                        for (int d = 0; d < DIM; ++d) gc[i * DIM + d] += qb[i] * Nf[d];
                }
            }
            if (vol[c] > 1e-15)
                for (int k = 0; k < NQ * DIM; ++k) gc[k] /= vol[c];
        });
    }

    // --------------------------------------------------------- reconstruct
    // LinearReconstructor::Reconstruct with VacuumLimiter + TVDLimiter, or PCM.
    void reconstruct(const T* q, const T* g, const double* xc, const double* xf, const T* qmin,
                     const T* qmax, T* out) const {
        if (st.reconstruction_order < 2) {
            for (int i = 0; i < NQ; ++i) out[i] = q[i];
            return;
        }
        T dx[3];
        for (int d = 0; d < DIM; ++d) dx[d] = xf[d] - xc[d];
        T qfu[NQ], delta[NQ];
        for (int i = 0; i < NQ; ++i) {
            delta[i] = 0.0;
            if (g)
                for (int d = 0; d < DIM; ++d) delta[i] += g[i * DIM + d] * dx[d];
            qfu[i] = q[i] + delta[i];
        }
        T fin[NQ];
        for (int i = 0; i < NQ; ++i) fin[i] = 1.0;
        if (st.limiter != ZSME_LIMITER_NONE) {
            // VacuumLimiter (tol 1e-2): h = component 1
            T tmp[NQ];
            for (int i = 0; i < NQ; ++i) tmp[i] = 1.0;
            if (NQ > 1 && qmin && qmin[1] < 1e-2)
                for (int i = 0; i < NQ; ++i) tmp[i] = 0.0;
            for (int i = 0; i < NQ; ++i) if (tmp[i] < fin[i]) fin[i] = tmp[i];
            // TVDLimiter (face-local Barth-Jespersen ratio)
            for (int i = 0; i < NQ; ++i) tmp[i] = 1.0;
            if (qmin && qmax) {
                for (int i = 0; i < NQ; ++i) {
                    T dq = qfu[i] - q[i];
                    if (std::abs(dq) < 1e-12) continue;
                    T al = 1.0;
                    if (dq > 0) {
                        if (qmax[i] > q[i]) al = std::min((T)1.0, (qmax[i] - q[i]) / dq);
                        else al = 0.0;
                    } else {
                        if (qmin[i] < q[i]) al = std::min((T)1.0, (qmin[i] - q[i]) / dq);
                        else al = 0.0;
                    }
                    tmp[i] = al;
                }
            }
            for (int i = 0; i < NQ; ++i) if (tmp[i] < fin[i]) fin[i] = tmp[i];
        }
        T alpha = 1.;
        for (int i = 0; i < NQ; ++i) if (alpha > fin[i]) alpha = fin[i];
        for (int i = 0; i < NQ; ++i) out[i] = q[i] + alpha * delta[i];
    }

    // ----------------------------------------------------- positivity (WB)
    // TransportStep::LimitGradientsWB (TransportStep.hpp:241-323): per cell,
    // Venkatakrishnan slopes on W = (b, eta = b + h, momenta) from the clamped
    // local state, dry cells first order, b and momentum slopes tied to eta,
    // the Zhang-Shu theta on the depth deviation (skipped under MOOD); the
    // effective gradients replace the raw ones (b slot: grad b_eff, h slot:
    // grad eta_eff, momenta: theta phi grad).
    void limit_gradients_wb(const std::vector<T>& xl, std::vector<T>& g) {
        const int B = 0, H = 1;
        const bool skip_theta = st.positivity == ZSME_POSITIVITY_MOOD;
        par_for(C, [&](int c, int) {
            T* gc = &g[(size_t)c * NQ * DIM];
            const T* qc = &xl[(size_t)c * NQ];
            T gr[NQ * DIM], geta[3], Wc[NQ], Wmin[NQ], Wmax[NQ], phi[NQ];
            for (int k = 0; k < NQ * DIM; ++k) gr[k] = gc[k];
            for (int d = 0; d < DIM; ++d) geta[d] = gr[H * DIM + d] + gr[B * DIM + d];
            const T h_bar = qc[H], b_bar = qc[B];
            for (int i = 0; i < NQ; ++i) Wc[i] = (i == H) ? (b_bar + h_bar) : qc[i];
            for (int i = 0; i < NQ; ++i) { Wmin[i] = Wc[i]; Wmax[i] = Wc[i]; }
            for (int k = nb_off[c]; k < nb_off[c + 1]; ++k) {
                const T* qn = &xl[(size_t)nb_list[k] * NQ];
                for (int i = 0; i < NQ; ++i) {
                    T w = (i == H) ? (qn[B] + qn[H]) : qn[i];
                    if (w < Wmin[i]) Wmin[i] = w;
                    if (w > Wmax[i]) Wmax[i] = w;
                }
            }
            // vol^(2/dim) (TransportStep.hpp:279), written exactly for dim 1 and 2
            const double eps2 = DIM == 2 ? vol[c] : DIM == 1 ? vol[c] * vol[c] : std::pow(vol[c], 2.0 / DIM);
            for (int i = 0; i < NQ; ++i) phi[i] = 1.0;
            for (int k = 0; k < K; ++k) {
                const int f = cf[(size_t)c * K + k];
                if (f < 0) continue;
                double r[3];
                for (int d = 0; d < DIM; ++d) r[d] = fc[2 * f + d] - cc[2 * c + d];
                for (int i = 0; i < NQ; ++i) {
                    T delta = 0.0;
                    for (int d = 0; d < DIM; ++d) delta += ((i == H) ? geta[d] : gr[i * DIM + d]) * r[d];
                    if (std::abs(delta) < 1e-14) continue;
                    T dm = (delta > 0) ? (Wmax[i] - Wc[i]) : (Wmin[i] - Wc[i]);
                    T num = dm * dm + eps2 + 2 * delta * dm, den = dm * dm + 2 * delta * delta + delta * dm + eps2;
                    T pf = (den > 1e-30) ? num / den : (T)1.0;
                    pf = std::max((T)0, std::min((T)1, pf));
                    if (pf < phi[i]) phi[i] = pf;
                }
            }
            if (h_bar < st.wet_dry_eps)
                for (int i = 0; i < NQ; ++i) phi[i] = 0.0;
            phi[B] = std::min(phi[B], phi[H]);
            for (int i = 0; i < NQ; ++i)
                if (i != B && i != H) phi[i] = std::min(phi[i], phi[H]);
            T sh[3];
            for (int d = 0; d < DIM; ++d) sh[d] = phi[H] * geta[d] - phi[B] * gr[B * DIM + d];
            T hmin = h_bar;
            for (int k = 0; k < K; ++k) {
                const int f = cf[(size_t)c * K + k];
                if (f < 0) continue;
                T hf = h_bar;
                for (int d = 0; d < DIM; ++d) hf += sh[d] * (fc[2 * f + d] - cc[2 * c + d]);
                if (hf < hmin) hmin = hf;
            }
            T theta = 1.0;
            if (!skip_theta && hmin < 0.0)
                theta = std::max((T)0, std::min((T)1, h_bar / std::max(h_bar - hmin, (T)1e-14)));
            for (int d = 0; d < DIM; ++d) {
                gc[B * DIM + d] = phi[B] * gr[B * DIM + d];
                gc[H * DIM + d] = phi[B] * gr[B * DIM + d] + theta * sh[d];
            }
            for (int i = 0; i < NQ; ++i)
                if (i != B && i != H)
                    for (int d = 0; d < DIM; ++d) gc[i * DIM + d] = theta * phi[i] * gr[i * DIM + d];
        });
    }

    // WBPositivityReconstructor::Reconstruct (Reconstruction.hpp:264-286):
    // eta_f and b_f from the effective gradients, h_f = max(eta_f - b_f, 0),
    // momenta zeroed where h_f < wet_dry_eps.
    void wb_reconstruct(const T* q, const T* g, const double* xc, const double* xf, T* out) const {
        const int B = 0, H = 1;
        T dx[3];
        for (int d = 0; d < DIM; ++d) dx[d] = xf[d] - xc[d];
        auto dot = [&](int slot) {
            T sum = 0.0;
            for (int d = 0; d < DIM; ++d) sum += g[slot * DIM + d] * dx[d];
            return sum;
        };
        const T b_bar = q[B], h_bar = q[H];
        const T b_f = b_bar + dot(B);
        const T eta_f = (b_bar + h_bar) + dot(H);
        const T h_f = std::max(eta_f - b_f, (T)0);
        for (int i = 0; i < NQ; ++i) {
            if (i == B) out[i] = b_f;
            else if (i == H) out[i] = h_f;
            else out[i] = (h_f < st.wet_dry_eps) ? (T)0 : (q[i] + dot(i));
        }
    }

    // The face reconstruction of the configured path.
    void recon(const T* q, const T* g, const double* xc, const double* xf, const T* qmin, const T* qmax,
               T* out) const {
        if (g && st.reconstruction_order >= 2 && st.positivity != ZSME_POSITIVITY_NONE)
            wb_reconstruct(q, g, xc, xf, out);
        else
            reconstruct(q, g, xc, xf, qmin, qmax, out);
    }

    // ------------------------------------------------------------- FormRHS
    void form_rhs(double t, const std::vector<T>& xg, std::vector<T>& f) {
        ph(zsme_flops::PREP);
        std::vector<T> xl = xg, al = A;          // local copies
        update_state_vec(xl, al);
        const bool o2 = st.reconstruction_order >= 2;
        std::vector<T> vmin, vmax;
        if (o2) {
            vmin.assign((size_t)C * NQ, 0.0);
            vmax.assign((size_t)C * NQ, 0.0);
par_for(C, [&](int c, int) {
                const T* q = &xl[(size_t)c * NQ];
                T* mn = &vmin[(size_t)c * NQ];
                T* mx = &vmax[(size_t)c * NQ];
                for (int i = 0; i < NQ; ++i) { mn[i] = q[i]; mx[i] = q[i]; }
                for (int k = nb_off[c]; k < nb_off[c + 1]; ++k) {
                    const T* qn = &xl[(size_t)nb_list[k] * NQ];
                    for (int i = 0; i < NQ; ++i) {
                        if (qn[i] < mn[i]) mn[i] = qn[i];
                        if (qn[i] > mx[i]) mx[i] = qn[i];
                    }
                }
            });
            // gradient of the UNCLAMPED global state (TransportStep.hpp:339)
            if (st.gradient == ZSME_GRADIENT_LSQ) gradient_lsq(xg, G); else gradient_gg(xg, G);
            if (st.positivity != ZSME_POSITIVITY_NONE) limit_gradients_wb(xl, G);
        }
        // per-face contributions: nc into L, nc into R, flux (all * area)
        std::vector<T> fb((size_t)F * 3 * NQ, 0.0);
        std::vector<char> active(F, 0);
par_for(F, [&](int f, int) {
            const double* Nf = &fn[2 * f];
            double area = 0;
            for (int d = 0; d < DIM; ++d) area += Nf[d] * Nf[d];
            area = std::sqrt(area);
            if (area <= 1e-15) return;
            T nh[3] = {0, 0, 0};
            for (int d = 0; d < DIM; ++d) nh[d] = Nf[d] / area;
            const T xf[3] = {fc[2 * f], fc[2 * f + 1], 0.0};
            int L = fcell[2 * f], R = fcell[2 * f + 1];
            T* ncL = &fb[(size_t)f * 3 * NQ];
            T* ncR = ncL + NQ;
            T* fl = ncR + NQ;
            if (R >= 0) {
                T qLf[NQ], qRf[NQ], aLf[NA], aRf[NA];
                ph(zsme_flops::PREP);
                recon(&xl[(size_t)L * NQ], o2 ? &G[(size_t)L * NQ * DIM] : nullptr, &cc[2 * L], &fc[2 * f],
                            o2 ? &vmin[(size_t)L * NQ] : nullptr, o2 ? &vmax[(size_t)L * NQ] : nullptr, qLf);
                recon(&xl[(size_t)R * NQ], o2 ? &G[(size_t)R * NQ * DIM] : nullptr, &cc[2 * R], &fc[2 * f],
                            o2 ? &vmin[(size_t)R * NQ] : nullptr, o2 ? &vmax[(size_t)R * NQ] : nullptr, qRf);
                ph(zsme_flops::FACE);
                for (int i = 0; i < NA; ++i) { aLf[i] = al[(size_t)L * NA + i]; aRf[i] = al[(size_t)R * NA + i]; }
                auto ra = M::update_aux_variables(qLf, aLf, params.data(), 0.0, xf);
                for (int i = 0; i < NA; ++i) aLf[i] = ra[i];
                auto rb = M::update_aux_variables(qRf, aRf, params.data(), 0.0, xf);
                for (int i = 0; i < NA; ++i) aRf[i] = rb[i];
                auto flux = N::numerical_flux(qLf, qRf, aLf, aRf, params.data(), nh);
                auto nc = N::numerical_fluctuations(qLf, qRf, aLf, aRf, params.data(), nh);
                for (int i = 0; i < NQ; ++i) {
                    ncL[i] = nc[NQ + i] * area;
                    ncR[i] = nc[i] * area;
                    fl[i] = flux[i] * area;
                }
                active[f] = 1;
            } else if (fbc[f] >= 0) {
                T qLf[NQ], aLf[NA], aRf[NA];
                ph(zsme_flops::PREP);
                recon(&xl[(size_t)L * NQ], o2 ? &G[(size_t)L * NQ * DIM] : nullptr, &cc[2 * L], &fc[2 * f],
                            o2 ? &vmin[(size_t)L * NQ] : nullptr, o2 ? &vmax[(size_t)L * NQ] : nullptr, qLf);
                ph(zsme_flops::FACE);
                for (int i = 0; i < NA; ++i) aLf[i] = al[(size_t)L * NA + i];
                auto ra = M::update_aux_variables(qLf, aLf, params.data(), t, xf);
                for (int i = 0; i < NA; ++i) aLf[i] = ra[i];
                auto qR = M::boundary_conditions(fbc[f], qLf, aLf, params.data(), nh, xf, t, 0.0);
                auto rb = M::update_aux_variables(qR.data, aLf, params.data(), t, xf);
                for (int i = 0; i < NA; ++i) aRf[i] = rb[i];
                auto flux = N::numerical_flux(qLf, qR.data, aLf, aRf, params.data(), nh);
                auto nc = N::numerical_fluctuations(qLf, qR.data, aLf, aRf, params.data(), nh);
                for (int i = 0; i < NQ; ++i) {
                    ncL[i] = nc[NQ + i] * area;
                    fl[i] = flux[i] * area;
                }
                active[f] = 2;
            }
        });
        // per cell: accumulate in increasing face order, then / volume
        ph(zsme_flops::GATHER);
        f.assign((size_t)C * NQ, 0.0);
par_for(C, [&](int c, int) {
            T* fcq = &f[(size_t)c * NQ];
            for (int k = 0; k < K; ++k) {
                int fi = cell_face_sorted[(size_t)c * K + k];
                if (fi < 0) break;
                if (!active[fi]) continue;
                const T* ncL = &fb[(size_t)fi * 3 * NQ];
                const T* ncR = ncL + NQ;
                const T* fl = ncR + NQ;
                if (fcell[2 * fi] == c) {
                    for (int i = 0; i < NQ; ++i) fcq[i] -= ncL[i];
                    for (int i = 0; i < NQ; ++i) fcq[i] -= fl[i];
                } else {
                    for (int i = 0; i < NQ; ++i) fcq[i] -= ncR[i];
                    for (int i = 0; i < NQ; ++i) fcq[i] += fl[i];
                }
            }
            if (vol[c] > 1e-15)
                for (int i = 0; i < NQ; ++i) fcq[i] /= vol[c];
        });
    }

    // ------------------------------------------------------------- source
    template <int n_q, int n_aux>
    static void aux_jacobian(const T* q, const T* aux, const T* p, T* J) {
        const T X0[3] = {0, 0, 0};
        if constexpr (zsme::HasAuxJacobian<M>::value) {
            auto r = M::update_aux_variables_jacobian_wrt_variables(q, aux, p);
            for (int i = 0; i < n_aux * n_q; ++i) J[i] = r[i];
        } else {
            for (int i = 0; i < n_aux * n_q; ++i) J[i] = 0;
            auto a0 = M::update_aux_variables(q, aux, p, 0.0, X0);
            T qp[n_q];
            for (int j = 0; j < n_q; ++j) {
                for (int m = 0; m < n_q; ++m) qp[m] = q[m];
                T h = (T)1e-7 * (std::abs(q[j]) + (T)1e-7);
                qp[j] += h;
                auto a1 = M::update_aux_variables(qp, aux, p, 0.0, X0);
                for (int k = 0; k < n_aux; ++k) J[k * n_q + j] = (a1[k] - a0[k]) / h;
            }
        }
    }
    static bool gepp(T* a, T* b, T* x) {
        const int n = NQ;
        for (int k = 0; k < n; ++k) {
            int mr = k;
            T mv = std::abs(a[k * n + k]);
            for (int i = k + 1; i < n; ++i)
                if (std::abs(a[i * n + k]) > mv) { mv = std::abs(a[i * n + k]); mr = i; }
            if (mv < 1e-14) return false;
            if (mr != k) {
                for (int j = k; j < n; ++j) std::swap(a[k * n + j], a[mr * n + j]);
                std::swap(b[k], b[mr]);
            }
            for (int i = k + 1; i < n; ++i) {
                T fct = a[i * n + k] / a[k * n + k];
                for (int j = k; j < n; ++j) a[i * n + j] -= fct * a[k * n + j];
                b[i] -= fct * b[k];
            }
        }
        for (int i = n - 1; i >= 0; --i) {
            T sum = 0.0;
            for (int j = i + 1; j < n; ++j) sum += a[i * n + j] * x[j];
            x[i] = (b[i] - sum) / a[i * n + i];
        }
        return true;
    }
    // SourceStep::SolveLocalCell; returns 1 if the iteration limit was hit.
    int solve_cell(T dtl, T* q, const T* aux_init) const {
        const T X0[3] = {0, 0, 0};
        T q_old[NQ], aux[NA], res[NQ], delta[NQ], J[NQ * NQ];
        for (int i = 0; i < NQ; ++i) q_old[i] = q[i];
        for (int i = 0; i < NA; ++i) aux[i] = aux_init[i];
        const T* p = params.data();
        int iter = 0;
        for (; iter < 15; ++iter) {
            auto ua = M::update_aux_variables(q, aux, p, 0.0, X0);
            for (int i = 0; i < NA; ++i) aux[i] = ua[i];
            auto S = M::source(q, aux, p, (T)0, dtl, X0);
            T rn = 0.0;
            for (int i = 0; i < NQ; ++i) {
                res[i] = q[i] - q_old[i] - dtl * S[i];
                rn += res[i] * res[i];
            }
            if (std::sqrt(rn) < 1e-8) break;
            auto dSdQ = M::source_jacobian_wrt_variables(q, aux, p);
            auto dSdA = M::source_jacobian_wrt_aux_variables(q, aux, p);
            T dAdQ[NA * NQ];
            aux_jacobian<NQ, NA>(q, aux, p, dAdQ);
            for (int i = 0; i < NQ * NQ; ++i) J[i] = 0.0;
            for (int i = 0; i < NQ; ++i) J[i * NQ + i] = 1.0;
            for (int i = 0; i < NQ; ++i)
                for (int j = 0; j < NQ; ++j) {
                    T term = dSdQ[i * NQ + j];
                    for (int k = 0; k < NA; ++k) term += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                    J[i * NQ + j] -= dtl * term;
                }
            for (int i = 0; i < NQ; ++i) res[i] = -res[i];
            if (gepp(J, res, delta)) {
                for (int i = 0; i < NQ; ++i) q[i] += delta[i];
            } else {
                break;
            }
        }
        return iter >= 15 ? 1 : 0;
    }
    // ---------------------------------------------------------------- IMEX
    // The implicit source of the IMEX strategy at state y: the state clamped and
    // its aux updated (UpdateState), the plugin's source there, zero in cells
    // with depth below 1e-6 (ModularSolver::AddImplicitSourceToResidual,
    // ModularSolver.hpp:82-124).
    void imex_source_cell(const T* y, const T* aux_init, T* S) const {
        const T X0[3] = {0, 0, 0};
        T ys[NQ], a[NA];
        for (int i = 0; i < NQ; ++i) ys[i] = y[i];
        for (int i = 0; i < NA; ++i) a[i] = aux_init[i];
        constrain_cell(ys, a);
        if (NQ > 1 && ys[1] < zsme::ark2e::dry_residual) {
            for (int i = 0; i < NQ; ++i) S[i] = 0.0;
            return;
        }
        auto r = M::source(ys, a, params.data(), (T)0, (T)0, X0);
        for (int i = 0; i < NQ; ++i) S[i] = r[i];
    }
    // One implicit stage of the IMEX step in one cell: y - z - hg S(y) = 0 by
    // Newton from y = z, the Jacobian I - hg (dS/dQ + dS/dAux dAux/dQ) at the
    // clamped state (the identity in cells drier than 1e-4,
    // ModularSolver::FormSourceJacobian, ModularSolver.hpp:403-460), the
    // elimination and the stopping rule of the source step (|residual| < 1e-8,
    // at most 15 updates).  Returns 1 when the update limit was hit.
    int imex_solve_cell(T hg, const T* z, T* y, const T* aux_init) const {
        T S[NQ], res[NQ], delta[NQ], J[NQ * NQ];
        for (int i = 0; i < NQ; ++i) y[i] = z[i];
        const T* p = params.data();
        int iter = 0;
        for (; iter < 15; ++iter) {
            imex_source_cell(y, aux_init, S);
            T rn = 0.0;
            for (int i = 0; i < NQ; ++i) {
                res[i] = y[i] - z[i] - hg * S[i];
                rn += res[i] * res[i];
            }
            if (std::sqrt(rn) < 1e-8) break;
            T ys[NQ], a[NA];
            for (int i = 0; i < NQ; ++i) ys[i] = y[i];
            for (int i = 0; i < NA; ++i) a[i] = aux_init[i];
            constrain_cell(ys, a);
            for (int i = 0; i < NQ * NQ; ++i) J[i] = 0.0;
            for (int i = 0; i < NQ; ++i) J[i * NQ + i] = 1.0;
            if (!(NQ > 1 && ys[1] < zsme::ark2e::dry_jacobian)) {
                auto dSdQ = M::source_jacobian_wrt_variables(ys, a, p);
                auto dSdA = M::source_jacobian_wrt_aux_variables(ys, a, p);
                T dAdQ[NA * NQ];
                aux_jacobian<NQ, NA>(ys, a, p, dAdQ);
                for (int i = 0; i < NQ; ++i)
                    for (int j = 0; j < NQ; ++j) {
                        T term = dSdQ[i * NQ + j];
                        for (int k = 0; k < NA; ++k) term += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                        J[i * NQ + j] -= hg * term;
                    }
            }
            for (int i = 0; i < NQ; ++i) res[i] = -res[i];
            if (!gepp(J, res, delta)) break;
            for (int i = 0; i < NQ; ++i) y[i] += delta[i];
        }
        return iter >= 15 ? 1 : 0;
    }
    // out = x + h (sum_j a_j G_j + sum_j at_j S_j), the terms added in order
    static void imex_combine(const std::vector<T>& x, T h, int n, const std::vector<T>* const* G, const double* a,
                             const std::vector<T>* const* S, const double* at, std::vector<T>& out) {
        out.resize(x.size());
        for (size_t k = 0; k < x.size(); ++k) {
            T acc = 0.0;
            for (int j = 0; j < n; ++j) acc += a[j] * (*G[j])[k];
            for (int j = 0; j < n; ++j) acc += at[j] * (*S[j])[k];
            out[k] = x[k] + h * acc;
        }
    }
    // The IMEX strategy's step (SolverStrategies.hpp:62-128: TSARKIMEX "2e",
    // transport explicit through FormRHS, source implicit) at the imposed dt h
    // without PETSc's step-size control: stage 0 is X; stages 1 and 2 solve
    // Y_i - h gamma S(Y_i) = Z_i per cell, their implicit derivative taken as
    // (Y_i - Z_i) / (h gamma); X <- X + h sum_j b_j (G_j + S_j).
    void imex_step(double t0, T h) {
        namespace K = zsme::ark2e;
        std::vector<T> G0, G1, G2, S0(X.size()), S1(X.size()), S2(X.size()), Z, Y1(X.size()), Y2(X.size());
        int nu = 0;
        form_rhs(t0, X, G0);
        par_for(C, [&](int c, int) { imex_source_cell(&X[(size_t)c * NQ], &A[(size_t)c * NA], &S0[(size_t)c * NQ]); });
        const T hg = h * K::gamma;
        auto stage = [&](std::vector<T>& Y, std::vector<T>& Si) {
            std::vector<int> part(par_width(C), 0);
            par_for(C, [&](int c, int t) {
                part[t] += imex_solve_cell(hg, &Z[(size_t)c * NQ], &Y[(size_t)c * NQ], &A[(size_t)c * NA]);
                for (int i = 0; i < NQ; ++i) {
                    const size_t id = (size_t)c * NQ + i;
                    Si[id] = (Y[id] - Z[id]) / hg;
                }
            });
            for (int v : part) nu += v;
        };
        {
            const std::vector<T>* G[1] = {&G0};
            const std::vector<T>* S[1] = {&S0};
            const double a[1] = {K::a10}, at[1] = {K::t10};
            imex_combine(X, h, 1, G, a, S, at, Z);
        }
        stage(Y1, S1);
        form_rhs(t0 + K::c1 * zsme::value(h), Y1, G1);
        {
            const std::vector<T>* G[2] = {&G0, &G1};
            const std::vector<T>* S[2] = {&S0, &S1};
            const double a[2] = {K::a20, K::a21}, at[2] = {K::t20, K::t21};
            imex_combine(X, h, 2, G, a, S, at, Z);
        }
        stage(Y2, S2);
        form_rhs(t0 + K::c2 * zsme::value(h), Y2, G2);
        {
            const std::vector<T>* G[3] = {&G0, &G1, &G2};
            const std::vector<T>* S[3] = {&S0, &S1, &S2};
            const double b[3] = {K::b0, K::b1, K::b2};
            std::vector<T> Xn;
            imex_combine(X, h, 3, G, b, S, b, Xn);
            X.swap(Xn);
        }
        n_unconv = nu;
    }

    void source_solve(T dtl) {
        std::vector<int> part(par_width(C), 0);
        par_for(C, [&](int c, int t) { part[t] += solve_cell(dtl, &X[(size_t)c * NQ], &A[(size_t)c * NA]); });
        int nu = 0;
        for (int v : part) nu += v;
        n_unconv = nu;
    }

    // ----------------------------------------------------- ComputeTimeStep
    double compute_dt() override {
        std::vector<double> part(par_width(C), std::numeric_limits<double>::max());
        par_for(C, [&](int c, int t) {
            double& best = part[t];
            const T* q = &X[(size_t)c * NQ];
            const T* a = &A[(size_t)c * NA];
            T eig = 0.0;
            for (int d = 0; d < DIM; ++d) {
                T n[3] = {0, 0, 0};
                n[d] = 1.0;
                auto r = N::local_max_abs_eigenvalue(q, a, params.data(), n);
                if (r[0] > eig) eig = r[0];
            }
            if (eig < 1e-14) return;
            if (!cfl_skip.empty() && cfl_skip[c]) return;   // a halo cell of a partition
            double rc = std::numeric_limits<double>::max();
            for (int k = 0; k < K; ++k) {
                int f = cf[(size_t)c * K + k];
                if (f < 0) continue;
                double d2 = 0.0;
                for (int d = 0; d < DIM; ++d) {
                    double dd = cc[2 * c + d] - fc[2 * f + d];
                    d2 += dd * dd;
                }
                double dist = std::sqrt(d2);
                if (dist < rc) rc = dist;
            }
            if (rc < std::numeric_limits<double>::max()) {
                double ratio = rc / zsme::value(eig);
                if (ratio < best) best = ratio;
            }
        });
        double best = std::numeric_limits<double>::max();
        for (double v : part) best = std::min(best, v);
        if (!std::isfinite(best) || best >= 0.5 * std::numeric_limits<double>::max()) return M::dt_max;
        return st.cfl * best;
    }

    // ------------------------------------------------- fully implicit strategy
    // SolverStrategies.hpp:133-195 (TSBDF order 2, IFunctionWrapper,
    // IJacobianWrapper with a matrix-free Jacobian and the assembled matrix as
    // the preconditioner's source) restated without PETSc: the residual and
    // the matrix blocks follow ModularSolver.hpp:82-124 and 238-371 operation
    // for operation; the Newton-Krylov iteration (Newton with backtracking,
    // left-preconditioned restarted GMRES with classical Gram-Schmidt, the
    // matrix's diagonal blocks as block-Jacobi preconditioner, Walker-Pernice
    // differencing) and BDF with variable-step coefficients are the same
    // algorithm as the GPU's, since PETSc's own SNES/KSP/TSAdapt histories
    // cannot be reproduced without PETSc.  Double precision only.
    bool imp_have_prev = false;
    double imp_h_prev = 0.0;
    int imp_stats_v[4] = {0, 0, 0, 0};
    std::vector<double> imp_xn, imp_xnm1;

    // f = (Xdot - S(x)) - R(x); xdot given, or (c0 x + c1 xn + c2 xnm1) / h
    void imp_residual(double t, const std::vector<double>& x, const double* xdot, const double* bdf,
                      const std::vector<double>* xn, const std::vector<double>* xnm1, std::vector<double>& f) {
        if constexpr (std::is_same<T, double>::value) {
            std::vector<double> R;
            form_rhs(t, x, R);
            f.resize(x.size());
            par_for(C, [&](int c, int) {
                double S[NQ];
                imex_source_cell(&x[(size_t)c * NQ], &A[(size_t)c * NA], S);
                for (int i = 0; i < NQ; ++i) {
                    const size_t id = (size_t)c * NQ + i;
                    const double xd = xdot ? xdot[id]
                                           : (bdf[0] * x[id] + bdf[1] * (*xn)[id] + bdf[2] * (*xnm1)[id]) / bdf[3];
                    f[id] = (xd - S[i]) - R[id];
                }
            });
        }
    }
    // ComputeFaceJacobian_FD / ComputeBoundaryJacobian_FD (ModularSolver.hpp:130-236)
    void imp_face_fd(const double* qL, const double* qR, const double* aL, const double* aR, const double* nh,
                     double* JLL, double* JLR, double* JRL, double* JRR) const {
        if constexpr (std::is_same<T, double>::value) {
            const double eps = 1e-7;
            const double X0[3] = {0, 0, 0};
            const double* p = params.data();
            auto Fb = N::numerical_flux(qL, qR, aL, aR, p, nh);
            auto NCb = N::numerical_fluctuations(qL, qR, aL, aR, p, nh);
            for (int j = 0; j < NQ; ++j) {
                double qp[NQ], ap[NA + 1];
                for (int k = 0; k < NQ; ++k) qp[k] = qL[k];
                for (int k = 0; k < NA; ++k) ap[k] = aL[k];
                qp[j] += eps;
                if (NA > 0) {
                    auto ra = M::update_aux_variables(qp, ap, p, 0.0, X0);
                    for (int k = 0; k < NA; ++k) ap[k] = ra[k];
                }
                auto Fp = N::numerical_flux(qp, qR, ap, aR, p, nh);
                auto NCp = N::numerical_fluctuations(qp, qR, ap, aR, p, nh);
                for (int i = 0; i < NQ; ++i) {
                    double dFlux = (Fp[i] - Fb[i]) / eps;
                    JLL[i * NQ + j] += dFlux;
                    JRL[i * NQ + j] -= dFlux;
                    JLL[i * NQ + j] += (NCp[NQ + i] - NCb[NQ + i]) / eps;
                    JRL[i * NQ + j] += (NCp[i] - NCb[i]) / eps;
                }
            }
            for (int j = 0; j < NQ; ++j) {
                double qp[NQ], ap[NA + 1];
                for (int k = 0; k < NQ; ++k) qp[k] = qR[k];
                for (int k = 0; k < NA; ++k) ap[k] = aR[k];
                qp[j] += eps;
                if (NA > 0) {
                    auto ra = M::update_aux_variables(qp, ap, p, 0.0, X0);
                    for (int k = 0; k < NA; ++k) ap[k] = ra[k];
                }
                auto Fp = N::numerical_flux(qL, qp, aL, ap, p, nh);
                auto NCp = N::numerical_fluctuations(qL, qp, aL, ap, p, nh);
                for (int i = 0; i < NQ; ++i) {
                    double dFlux = (Fp[i] - Fb[i]) / eps;
                    JLR[i * NQ + j] += dFlux;
                    JRR[i * NQ + j] -= dFlux;
                    JLR[i * NQ + j] += (NCp[NQ + i] - NCb[NQ + i]) / eps;
                    JRR[i * NQ + j] += (NCp[i] - NCb[i]) / eps;
                }
            }
        }
    }
    void imp_boundary_fd(const double* qL, const double* aL, const double* nh, const double* xf, double t, int bc,
                         double* JLL) const {
        if constexpr (std::is_same<T, double>::value) {
            const double eps = 1e-7;
            const double* p = params.data();
            auto qRb = M::boundary_conditions(bc, qL, aL, p, nh, xf, t, 0.0);
            double aRb[NA + 1];
            if (NA > 0) {
                auto ra = M::update_aux_variables(qRb.data, aL, p, t, xf);
                for (int k = 0; k < NA; ++k) aRb[k] = ra[k];
            }
            auto Fb = N::numerical_flux(qL, qRb.data, aL, aRb, p, nh);
            auto NCb = N::numerical_fluctuations(qL, qRb.data, aL, aRb, p, nh);
            for (int j = 0; j < NQ; ++j) {
                double qp[NQ], ap[NA + 1], ar[NA + 1];
                for (int k = 0; k < NQ; ++k) qp[k] = qL[k];
                for (int k = 0; k < NA; ++k) ap[k] = aL[k];
                qp[j] += eps;
                if (NA > 0) {
                    auto ra = M::update_aux_variables(qp, ap, p, t, xf);
                    for (int k = 0; k < NA; ++k) ap[k] = ra[k];
                }
                auto qr = M::boundary_conditions(bc, qp, ap, p, nh, xf, t, 0.0);
                if (NA > 0) {
                    auto ra = M::update_aux_variables(qr.data, ap, p, t, xf);
                    for (int k = 0; k < NA; ++k) ar[k] = ra[k];
                }
                auto Fp = N::numerical_flux(qp, qr.data, ap, ar, p, nh);
                auto NCp = N::numerical_fluctuations(qp, qr.data, ap, ar, p, nh);
                for (int i = 0; i < NQ; ++i) {
                    double dFlux = (Fp[i] - Fb[i]) / eps;
                    JLL[i * NQ + j] += dFlux;
                    JLL[i * NQ + j] += (NCp[NQ + i] - NCb[NQ + i]) / eps;
                }
            }
        }
    }
    // FormImplicitJacobian (ModularSolver.hpp:238-371) at (t, x, a): Pd [C][NQ NQ]
    // diagonal blocks, Po [F][2][NQ NQ] the (L, R) and (R, L) blocks; entries
    // start at zero and take the source blocks, then the faces in order
    void imp_assemble(double t, const std::vector<double>& xg, double a, std::vector<double>& Pd,
                      std::vector<double>& Po) {
        if constexpr (std::is_same<T, double>::value) {
            constexpr int Q2 = NQ * NQ;
            std::vector<double> xl = xg, al = A;
            update_state_vec(xl, al);
            Pd.assign((size_t)C * Q2, 0.0);
            Po.assign((size_t)F * 2 * Q2, 0.0);
            const double* p = params.data();
            par_for(C, [&](int c, int) {
                const double* qc = &xl[(size_t)c * NQ];
                const double* ac = &al[(size_t)c * NA];
                double J[Q2];
                if (NQ > 1 && qc[1] < 1e-4) {
                    for (int e = 0; e < Q2; ++e) J[e] = 0.0;
                    for (int i = 0; i < NQ; ++i) J[i * NQ + i] = a;
                } else {
                    auto dSdQ = M::source_jacobian_wrt_variables(qc, ac, p);
                    auto dSdA = M::source_jacobian_wrt_aux_variables(qc, ac, p);
                    double dAdQ[NA * NQ + 1];
                    aux_jacobian<NQ, NA>(qc, ac, p, dAdQ);
                    for (int i = 0; i < NQ; ++i)
                        for (int j = 0; j < NQ; ++j) {
                            double val = i == j ? a : 0.0;
                            double dSource = dSdQ[i * NQ + j];
                            for (int k = 0; k < NA; ++k) dSource += dSdA[i * NA + k] * dAdQ[k * NQ + j];
                            J[i * NQ + j] = val - dSource;
                        }
                }
                for (int e = 0; e < Q2; ++e) Pd[(size_t)c * Q2 + e] += J[e];
            });
            for (int f = 0; f < F; ++f) {
                double area = 0;
                for (int d = 0; d < DIM; ++d) area += fn[2 * f + d] * fn[2 * f + d];
                area = std::sqrt(area);
                if (area <= 1e-15) continue;
                double nh[3] = {0, 0, 0};
                for (int d = 0; d < DIM; ++d) nh[d] = fn[2 * f + d] / area;
                const int L = fcell[2 * f], R = fcell[2 * f + 1];
                const double* qL = &xl[(size_t)L * NQ];
                const double* aL = &al[(size_t)L * NA];
                if (R >= 0) {
                    double JLL[Q2] = {0}, JLR[Q2] = {0}, JRL[Q2] = {0}, JRR[Q2] = {0};
                    imp_face_fd(qL, &xl[(size_t)R * NQ], aL, &al[(size_t)R * NA], nh, JLL, JLR, JRL, JRR);
                    const double fL = area / vol[L], fR = area / vol[R];
                    for (int e = 0; e < Q2; ++e) {
                        JLL[e] *= fL; JLR[e] *= fL;
                        JRL[e] *= fR; JRR[e] *= fR;
                    }
                    for (int e = 0; e < Q2; ++e) Pd[(size_t)L * Q2 + e] += JLL[e];
                    for (int e = 0; e < Q2; ++e) Po[((size_t)f * 2 + 0) * Q2 + e] += JLR[e];
                    for (int e = 0; e < Q2; ++e) Po[((size_t)f * 2 + 1) * Q2 + e] += JRL[e];
                    for (int e = 0; e < Q2; ++e) Pd[(size_t)R * Q2 + e] += JRR[e];
                } else if (fbc[f] >= 0) {
                    double JLL[Q2] = {0};
                    const double xf[3] = {fc[2 * f], fc[2 * f + 1], 0.0};
                    imp_boundary_fd(qL, aL, nh, xf, t, fbc[f], JLL);
                    const double fL = area / vol[L];
                    for (int e = 0; e < Q2; ++e) JLL[e] *= fL;
                    for (int e = 0; e < Q2; ++e) Pd[(size_t)L * Q2 + e] += JLL[e];
                }
            }
        }
    }
    // LU with partial pivoting of every diagonal block (identity where a pivot
    // vanishes), and the block solve z = D^-1 r
    static void imp_block_lu(std::vector<double>& lu, std::vector<int>& piv, int C) {
        constexpr int Q2 = NQ * NQ;
        piv.assign((size_t)C * NQ, 0);
        par_for(C, [&](int c, int) {
            double* A_ = &lu[(size_t)c * Q2];
            int* pv = &piv[(size_t)c * NQ];
            bool ok = true;
            for (int k = 0; k < NQ; ++k) {
                int mr = k;
                double mv = std::fabs(A_[k * NQ + k]);
                for (int i = k + 1; i < NQ; ++i) {
                    const double v = std::fabs(A_[i * NQ + k]);
                    if (v > mv) { mv = v; mr = i; }
                }
                pv[k] = mr;
                if (mr != k)
                    for (int j = 0; j < NQ; ++j) std::swap(A_[k * NQ + j], A_[mr * NQ + j]);
                const double pkk = A_[k * NQ + k];
                if (!(mv > 0.0) || !std::isfinite(pkk)) { ok = false; break; }
                for (int i = k + 1; i < NQ; ++i) {
                    const double l = A_[i * NQ + k] / pkk;
                    A_[i * NQ + k] = l;
                    for (int j = k + 1; j < NQ; ++j) A_[i * NQ + j] -= l * A_[k * NQ + j];
                }
            }
            if (!ok) {
                for (int e = 0; e < Q2; ++e) A_[e] = 0.0;
                for (int i = 0; i < NQ; ++i) { A_[i * NQ + i] = 1.0; pv[i] = i; }
            }
        });
    }
    static void imp_block_solve(const std::vector<double>& lu, const std::vector<int>& piv, int C,
                                std::vector<double>& z) {
        constexpr int Q2 = NQ * NQ;
        par_for(C, [&](int c, int) {
            const double* A_ = &lu[(size_t)c * Q2];
            const int* pv = &piv[(size_t)c * NQ];
            double* b = &z[(size_t)c * NQ];
            for (int k = 0; k < NQ; ++k) {
                const int mr = pv[k];
                if (mr != k) std::swap(b[k], b[mr]);
                for (int i = k + 1; i < NQ; ++i) b[i] -= A_[i * NQ + k] * b[k];
            }
            for (int i = NQ - 1; i >= 0; --i) {
                double s = b[i];
                for (int j = i + 1; j < NQ; ++j) s -= A_[i * NQ + j] * b[j];
                b[i] = s / A_[i * NQ + i];
            }
        });
    }
    static double imp_dot(const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
        return s;
    }
    // One BDF step of size h (the GPU's algorithm; see the header comment);
    // false when Newton did not converge (the state is then the step's start)
    bool imp_step(double t0, double h) {
        if constexpr (std::is_same<T, double>::value) {
            const size_t n = X.size();
            if (imp_have_prev) std::swap(imp_xn, imp_xnm1);
            imp_xn = X;
            double bdf[4] = {1.0, -1.0, 0.0, h};
            const std::vector<double>* xnm1 = &imp_xn;
            if (imp_have_prev) {
                const double w = h / imp_h_prev;
                bdf[0] = (1.0 + 2.0 * w) / (1.0 + w);
                bdf[1] = -(1.0 + w);
                bdf[2] = w * w / (1.0 + w);
                xnm1 = &imp_xnm1;
            }
            const double shift = bdf[0] / h, t1 = t0 + h;
            auto resid = [&](const std::vector<double>& x, std::vector<double>& f) {
                imp_residual(t1, x, nullptr, bdf, &imp_xn, xnm1, f);
            };
            std::vector<double> Fv, Ft, Pd, Po, lu, xt(n), d(n), w(n), r0(n), r(n);
            std::vector<int> piv;
            resid(X, Fv);
            double fnorm = std::sqrt(imp_dot(Fv, Fv));
            const double fnorm0 = fnorm;
            int it = 0, gm_total = 0, halvings = 0, conv = 0;
            constexpr int m = 30;
            for (; it < 50; ++it) {
                if (fnorm <= 1e-4 || (it > 0 && fnorm <= 1e-3 * fnorm0)) { conv = 1; break; }
                if (!std::isfinite(fnorm)) break;
                const double xnorm = std::sqrt(imp_dot(X, X));
                imp_assemble(t1, X, shift, Pd, Po);
                lu = Pd;
                imp_block_lu(lu, piv, C);
                // M^-1 J v by differencing
                auto apply = [&](const std::vector<double>& v, std::vector<double>& out) {
                    const double vnorm = std::sqrt(imp_dot(v, v));
                    out.assign(n, 0.0);
                    if (!(vnorm > 0.0)) return;
                    const double hv = 1.4901161193847656e-08 * std::sqrt(1.0 + xnorm) / vnorm;
                    for (size_t i = 0; i < n; ++i) xt[i] = 1.0 * X[i] + hv * v[i];
                    resid(xt, Ft);
                    for (size_t i = 0; i < n; ++i) out[i] = (Ft[i] - Fv[i]) / hv;
                    imp_block_solve(lu, piv, C, out);
                };
                // GMRES
                int gm = 0;
                std::fill(d.begin(), d.end(), 0.0);
                for (size_t i = 0; i < n; ++i) r0[i] = -1.0 * Fv[i];
                imp_block_solve(lu, piv, C, r0);
                double beta = std::sqrt(imp_dot(r0, r0));
                if (beta > 0.0) {
                    const double tol = std::max(1e-5 * beta, 1e-50);
                    std::vector<std::vector<double>> V(m + 1, std::vector<double>(n));
                    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
                    const std::vector<double>* rp = &r0;
                    while (true) {
                        for (size_t i = 0; i < n; ++i) V[0][i] = (1.0 / beta) * (*rp)[i];
                        std::fill(g.begin(), g.end(), 0.0);
                        g[0] = beta;
                        int j = 0;
                        bool done = false;
                        for (; j < m;) {
                            apply(V[j], w);
                            double hcol[m + 1];
                            for (int i = 0; i <= j; ++i) hcol[i] = imp_dot(V[i], w);
                            for (size_t e = 0; e < n; ++e) {
                                double s = w[e];
                                for (int i = 0; i <= j; ++i) s -= hcol[i] * V[i][e];
                                w[e] = s;
                            }
                            const double hn = std::sqrt(imp_dot(w, w));
                            if (hn > 0.0)
                                for (size_t e = 0; e < n; ++e) V[j + 1][e] = (1.0 / hn) * w[e];
                            for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
                            H[(size_t)(j + 1) * m + j] = hn;
                            for (int i = 0; i < j; ++i) {
                                const double a0 = H[(size_t)i * m + j], a1 = H[(size_t)(i + 1) * m + j];
                                H[(size_t)i * m + j] = cs[i] * a0 + sn[i] * a1;
                                H[(size_t)(i + 1) * m + j] = -sn[i] * a0 + cs[i] * a1;
                            }
                            const double hjj = H[(size_t)j * m + j], hj1 = H[(size_t)(j + 1) * m + j];
                            const double den = std::sqrt(hjj * hjj + hj1 * hj1);
                            cs[j] = den > 0.0 ? hjj / den : 1.0;
                            sn[j] = den > 0.0 ? hj1 / den : 0.0;
                            H[(size_t)j * m + j] = den;
                            H[(size_t)(j + 1) * m + j] = 0.0;
                            g[j + 1] = -sn[j] * g[j];
                            g[j] = cs[j] * g[j];
                            ++gm;
                            ++j;
                            const double res = std::fabs(g[j]);
                            if (res <= tol || !(hn > 0.0) || gm >= 10000 || !std::isfinite(res)) {
                                done = true;
                                break;
                            }
                        }
                        for (int i = j - 1; i >= 0; --i) {
                            double s = g[i];
                            for (int k = i + 1; k < j; ++k) s -= H[(size_t)i * m + k] * y[k];
                            y[i] = H[(size_t)i * m + i] != 0.0 ? s / H[(size_t)i * m + i] : 0.0;
                        }
                        for (size_t e = 0; e < n; ++e) {
                            double s = d[e];
                            for (int k = 0; k < j; ++k) s += y[k] * V[k][e];
                            d[e] = s;
                        }
                        if (done) break;
                        apply(d, w);
                        for (size_t e = 0; e < n; ++e) r[e] = 1.0 * r0[e] + -1.0 * w[e];
                        rp = &r;
                        beta = std::sqrt(imp_dot(r, r));
                        if (!(beta > tol)) break;
                    }
                }
                gm_total += gm;
                // backtracking
                double lambda = 1.0, ft = 0.0;
                bool descent = false;
                for (int ls = 0; ls < 10; ++ls) {
                    for (size_t i = 0; i < n; ++i) xt[i] = 1.0 * X[i] + lambda * d[i];
                    resid(xt, Ft);
                    ft = std::sqrt(imp_dot(Ft, Ft));
                    if (ft <= (1.0 - 1e-4 * lambda) * fnorm) { descent = true; break; }
                    lambda *= 0.5;
                    ++halvings;
                }
                if (!descent) break;
                X = xt;
                Fv = Ft;
                fnorm = ft;
                const double dnorm = std::sqrt(imp_dot(d, d)), xn2 = std::sqrt(imp_dot(X, X));
                if (lambda * dnorm <= 1e-8 * xn2) { conv = fnorm <= 1e-4 || fnorm <= 1e-3 * fnorm0 ? 1 : 2; ++it; break; }
            }
            imp_stats_v[0] = it;
            imp_stats_v[1] = gm_total;
            imp_stats_v[2] = halvings;
            imp_stats_v[3] = conv;
            if (!conv) {   // nothing of the step is kept; the driver stops
                X = imp_xn;
                if (imp_have_prev) std::swap(imp_xn, imp_xnm1);
                return false;
            }
            imp_h_prev = h;
            imp_have_prev = true;
        }
        return true;
    }
    int implicit_stats(int* out) const override {
        for (int i = 0; i < 4; ++i) out[i] = imp_stats_v[i];
        return 0;
    }
    void implicit_function(double t, const double* x, const double* xdot, double* f) override {
        if constexpr (std::is_same<T, double>::value) {
            std::vector<double> xv(x, x + (size_t)C * NQ), fv;
            imp_residual(t, xv, xdot, nullptr, nullptr, nullptr, fv);
            for (size_t i = 0; i < fv.size(); ++i) f[i] = fv[i];
        }
    }
    void implicit_jacobian(double t, const double* x, double a, double* diag, double* faces) override {
        if constexpr (std::is_same<T, double>::value) {
            std::vector<double> xv(x, x + (size_t)C * NQ), Pd, Po;
            imp_assemble(t, xv, a, Pd, Po);
            if (diag) std::copy(Pd.begin(), Pd.end(), diag);
            if (faces) std::copy(Po.begin(), Po.end(), faces);
        }
    }

    // ------------------------------------------------------------ driver
    void set_state(const double* q, double t) override {
        imp_have_prev = false;
        X.assign(q, q + (size_t)C * NQ);
        std::fill(A.begin(), A.end(), 0.0);
        time = t;
        update_state_vec(X, A);                                  // MUSCLSolver.hpp:54
        dt = std::max(compute_dt(), st.min_dt);                  // MUSCLSolver.hpp:103
    }
    static void values(const std::vector<T>& v, double* out) {
        for (size_t i = 0; i < v.size(); ++i) out[i] = zsme::value(v[i]);
    }
    void get_state(double* q) const override { values(X, q); }
    void get_aux(double* a) const override { values(A, a); }
    void get_time(double* t, double* d) const override { *t = time; *d = dt; }
    void rhs(double t, const double* x, double* f) override {
        std::vector<T> xv(x, x + (size_t)C * NQ), fv;
        form_rhs(t, xv, fv);
        values(fv, f);
    }
    void gradient(const double* x, double* g) override {
        std::vector<T> xv(x, x + (size_t)C * NQ), gv((size_t)C * NQ * DIM);
        if (st.gradient == ZSME_GRADIENT_LSQ) gradient_lsq(xv, gv); else gradient_gg(xv, gv);
        values(gv, g);
    }
    // Seed the tangent direction of the (constrained) state and of the
    // parameters; read the state's tangent.  Dual<1> instances only.
    void set_tangent(const double* dq, const double* dp) override {
        if constexpr (std::is_same<T, zsme::Dual<1>>::value) {
            for (size_t i = 0; i < X.size(); ++i) X[i].d[0] = dq ? dq[i] : 0.0;
            for (size_t k = 0; k < params.size(); ++k) params[k].d[0] = dp ? dp[k] : 0.0;
        }
    }
    void get_tangent(double* dq) const override {
        if constexpr (std::is_same<T, zsme::Dual<1>>::value)
            for (size_t i = 0; i < X.size(); ++i) dq[i] = X[i].d[0];
    }
    void update_state() override { update_state_vec(X, A); }
    void source(double d) override { source_solve(d); }

    // TSStep: SSP-RK(s,2) for order >= 2, forward Euler for order 1.
    void ts_step(double t0, double h) {
        std::vector<T> F;
        const size_t n = X.size();
        if (st.reconstruction_order < 2) {
            form_rhs(t0, X, F);
            ph(zsme_flops::GATHER);
            for (size_t i = 0; i < n; ++i) X[i] = X[i] + h * F[i];
            return;
        }
        const int s = st.ssp_stages;
        std::vector<T> w = X;
        for (int i = 0; i < s - 1; ++i) {
            double stage_time = t0 + h * (i / (s - 1.));
            form_rhs(stage_time, w, F);
            ph(zsme_flops::GATHER);
            const double a = h / (s - 1.);
            for (size_t k = 0; k < n; ++k) w[k] = w[k] + a * F[k];
        }
        form_rhs(t0 + h, w, F);
        ph(zsme_flops::GATHER);
        const double al = (s - 1.) / s, be = h / s, ga = 1. / s;
        for (size_t k = 0; k < n; ++k) X[k] = al * w[k] + be * F[k] + ga * X[k];
    }
    // Local MOOD (MUSCLSolver.hpp:130-171, 197-229; TransportStep.hpp:363-381):
    // cells whose depth ends below -1e-10 are overwritten by the first-order
    // forward-Euler update from the step's start state Xs (piecewise constant
    // states, fluxes of the faces touching a troubled cell), then the
    // constraints are applied again.
    void mood_override(double t0, double d0, const std::vector<T>& Xs) {
        std::vector<char> bad(C, 0);
        int nt = 0;
        for (int c = 0; c < C; ++c)
            if (X[(size_t)c * NQ + 1] < -1.0e-10) { bad[c] = 1; ++nt; }
        if (!nt) return;
        n_troubled += nt;
        std::vector<T> xl = Xs, al = A;
        update_state_vec(xl, al);
        std::vector<T> fb((size_t)F * 3 * NQ, 0.0);
        std::vector<char> active(F, 0);
        par_for(F, [&](int f, int) {
            const int L = fcell[2 * f], R = fcell[2 * f + 1];
            if (!(bad[L] || (R >= 0 && bad[R]))) return;
            const double* Nf = &fn[2 * f];
            double area = 0;
            for (int d = 0; d < DIM; ++d) area += Nf[d] * Nf[d];
            area = std::sqrt(area);
            if (area <= 1e-15) return;
            T nh[3] = {0, 0, 0};
            for (int d = 0; d < DIM; ++d) nh[d] = Nf[d] / area;
            const T xf[3] = {fc[2 * f], fc[2 * f + 1], 0.0};
            T* ncL = &fb[(size_t)f * 3 * NQ];
            T* ncR = ncL + NQ;
            T* fl = ncR + NQ;
            T qLf[NQ], aLf[NA], aRf[NA];
            for (int i = 0; i < NQ; ++i) qLf[i] = xl[(size_t)L * NQ + i];
            for (int i = 0; i < NA; ++i) aLf[i] = al[(size_t)L * NA + i];
            if (R >= 0) {
                T qRf[NQ];
                for (int i = 0; i < NQ; ++i) qRf[i] = xl[(size_t)R * NQ + i];
                for (int i = 0; i < NA; ++i) aRf[i] = al[(size_t)R * NA + i];
                auto ra = M::update_aux_variables(qLf, aLf, params.data(), 0.0, xf);
                for (int i = 0; i < NA; ++i) aLf[i] = ra[i];
                auto rb = M::update_aux_variables(qRf, aRf, params.data(), 0.0, xf);
                for (int i = 0; i < NA; ++i) aRf[i] = rb[i];
                auto flux = N::numerical_flux(qLf, qRf, aLf, aRf, params.data(), nh);
                auto nc = N::numerical_fluctuations(qLf, qRf, aLf, aRf, params.data(), nh);
                for (int i = 0; i < NQ; ++i) {
                    ncL[i] = nc[NQ + i] * area;
                    ncR[i] = nc[i] * area;
                    fl[i] = flux[i] * area;
                }
                active[f] = 1;
            } else if (fbc[f] >= 0) {
                auto ra = M::update_aux_variables(qLf, aLf, params.data(), t0, xf);
                for (int i = 0; i < NA; ++i) aLf[i] = ra[i];
                auto qR = M::boundary_conditions(fbc[f], qLf, aLf, params.data(), nh, xf, t0, 0.0);
                auto rb = M::update_aux_variables(qR.data, aLf, params.data(), t0, xf);
                for (int i = 0; i < NA; ++i) aRf[i] = rb[i];
                auto flux = N::numerical_flux(qLf, qR.data, aLf, aRf, params.data(), nh);
                auto nc = N::numerical_fluctuations(qLf, qR.data, aLf, aRf, params.data(), nh);
                for (int i = 0; i < NQ; ++i) {
                    ncL[i] = nc[NQ + i] * area;
                    fl[i] = flux[i] * area;
                }
                active[f] = 2;
            }
        });
        par_for(C, [&](int c, int) {
            if (!bad[c]) return;
            T fcq[NQ];
            for (int i = 0; i < NQ; ++i) fcq[i] = 0.0;
            for (int k = 0; k < K; ++k) {
                const int fi = cell_face_sorted[(size_t)c * K + k];
                if (fi < 0) break;
                if (!active[fi]) continue;
                const T* ncL = &fb[(size_t)fi * 3 * NQ];
                const T* ncR = ncL + NQ;
                const T* fl = ncR + NQ;
                if (fcell[2 * fi] == c) {
                    for (int i = 0; i < NQ; ++i) fcq[i] -= ncL[i];
                    for (int i = 0; i < NQ; ++i) fcq[i] -= fl[i];
                } else {
                    for (int i = 0; i < NQ; ++i) fcq[i] -= ncR[i];
                    for (int i = 0; i < NQ; ++i) fcq[i] += fl[i];
                }
            }
            if (vol[c] > 1e-15)
                for (int i = 0; i < NQ; ++i) fcq[i] /= vol[c];
            for (int i = 0; i < NQ; ++i) X[(size_t)c * NQ + i] = Xs[(size_t)c * NQ + i] + d0 * fcq[i];
        });
        update_state_vec(X, A);
    }

    void step(int nsteps, const double* dts) override {
        for (int it = 0; it < nsteps; ++it) {
            if (!(time < st.t_end)) break;
            double t0 = time;
            double d0 = dts ? dts[it] : dt;
            if (t0 + d0 > st.t_end) d0 = st.t_end - t0;
            const bool mood = st.positivity == ZSME_POSITIVITY_MOOD;
            std::vector<T> Xs;
            if (mood) Xs = X;
            const bool imex = st.time_integration == ZSME_TIME_IMEX;
            const bool implicit = st.time_integration == ZSME_TIME_IMPLICIT;
            if (imex) imex_step(t0, d0);
            else if (implicit) {
                if (!imp_step(t0, d0)) break;   // Newton failed: the step is not taken
            } else {
                ts_step(t0, d0);
            }
            ph(zsme_flops::FINAL);
            time = t0 + d0;
            update_state_vec(X, A);                            // EnforcePhysicalConstraints
            if (mood) mood_override(t0, d0, Xs);
            if (st.source && !imex && !implicit) {             // IMEX and implicit carry the source
                source_solve(d0);
                update_state_vec(X, A);
            }
            update_state_vec(X, A);                            // PostStep
            dt = compute_dt();
        }
    }
};

// Pointwise evaluation of one plugin function (for pinning the generated
// headers against the reference's).  fn: 0 numerical_flux, 1
// numerical_fluctuations, 2 local_max_abs_eigenvalue, 3 source, 4
// source_jacobian_wrt_variables, 5 source_jacobian_wrt_aux_variables, 6
// update_variables, 7 update_aux_variables, 8 boundary_conditions(bc 0),
// 9 eigenvalues, 10 flux, 11 solver-side dAux/dQ (SourceStep.hpp:26-53),
// 12 nonconservative_matrix, 13 the Jacobian of [numerical_flux,
// numerical_fluctuations] (3 nq rows) with respect to [qL, qR] (2 nq
// columns), row-major, by dual numbers.
template <template <typename> class MT, template <typename> class NT>
int pointwise(int fn, const double* qL, const double* qR, const double* aL, const double* aR,
              const double* p, const double* n, double s, double* out) {
    using M = MT<double>;
    using N = NT<double>;
    const double X0[3] = {0, 0, 0};
    auto put = [&](const auto& r, int k) { for (int i = 0; i < k; ++i) out[i] = r[i]; return k; };
    constexpr int nq = M::n_dof_q, na = M::n_dof_qaux, dim = M::dimension;
    switch (fn) {
        case 0: return put(N::numerical_flux(qL, qR, aL, aR, p, n), nq);
        case 1: return put(N::numerical_fluctuations(qL, qR, aL, aR, p, n), 2 * nq);
        case 2: return put(N::local_max_abs_eigenvalue(qL, aL, p, n), 1);
        case 3: return put(M::source(qL, aL, p, 0.0, s, X0), nq);
        case 4: return put(M::source_jacobian_wrt_variables(qL, aL, p), nq * nq);
        case 5: return put(M::source_jacobian_wrt_aux_variables(qL, aL, p), nq * na);
        case 6: return put(M::update_variables(qL, aL, p, s), nq);
        case 7: return put(M::update_aux_variables(qL, aL, p, 0.0, X0), na);
        case 8: return put(M::boundary_conditions(0, qL, aL, p, n, X0, 0.0, 0.0), nq);
        case 9: return put(M::eigenvalues(qL, aL, p, n), nq);
        case 10: return put(M::flux(qL, aL, p), nq * dim);
        case 11: {
            double J[na * nq];
            Oracle<MT, NT>::template aux_jacobian<nq, na>(qL, aL, p, J);
            for (int i = 0; i < na * nq; ++i) out[i] = J[i];
            return na * nq;
        }
        case 12: return put(M::nonconservative_matrix(qL, aL, p), nq * nq * dim);
        case 13: {
            using D = zsme::Dual<nq>;
            for (int side = 0; side < 2; ++side) {
                D dl[nq], dr[nq], dal[na], dar[na], dp[M::n_parameters], dn[3];
                for (int i = 0; i < nq; ++i) {
                    dl[i] = side == 0 ? D::seed(qL[i], i) : D(qL[i]);
                    dr[i] = side == 1 ? D::seed(qR[i], i) : D(qR[i]);
                }
                for (int i = 0; i < na; ++i) { dal[i] = D(aL[i]); dar[i] = D(aR[i]); }
                for (int i = 0; i < M::n_parameters; ++i) dp[i] = D(p[i]);
                for (int i = 0; i < 3; ++i) dn[i] = D(n[i]);
                const auto fl = NT<D>::numerical_flux(dl, dr, dal, dar, dp, dn);
                const auto nc = NT<D>::numerical_fluctuations(dl, dr, dal, dar, dp, dn);
                for (int r = 0; r < 3 * nq; ++r)
                    for (int j = 0; j < nq; ++j)
                        out[r * 2 * nq + side * nq + j] = r < nq ? fl[r].d[j] : nc[r - nq].d[j];
            }
            return 6 * nq * nq;
        }
    }
    return -1;
}

// The generated reverse-mode face derivative, or -1 where the plugin has none.
template <template <typename> class MT, template <typename> class NT>
int flux_vjp(const double* qL, const double* qR, const double* aL, const double* aR, const double* p,
             const double* n, const double* w, double* g) {
    if constexpr (zsme::HasFluxVJP<NT<double>>::value) {
        NT<double>::numerical_flux_fluct_vjp(qL, qR, aL, aR, p, n, w, g);
        return 2 * MT<double>::n_dof_q;
    } else {
        return -1;
    }
}

struct Entry {
    const char* name;
    OracleBase* (*make)(const zsme_mesh*, const zsme_settings*, const double*);
    int (*pw)(int, const double*, const double*, const double*, const double*, const double*,
              const double*, double, double*);
    int (*vjp)(const double*, const double*, const double*, const double*, const double*, const double*,
               const double*, double*);
    int nq, na, np, dim;
    OracleBase* (*make_tlm)(const zsme_mesh*, const zsme_settings*, const double*);
    OracleBase* (*make_counting)(const zsme_mesh*, const zsme_settings*, const double*);
};

template <template <typename> class MT, template <typename> class NT>
OracleBase* make_oracle(const zsme_mesh* m, const zsme_settings* s, const double* p) {
    return new Oracle<MT, NT>(m, s, p);
}
template <template <typename> class MT, template <typename> class NT>
OracleBase* make_tlm(const zsme_mesh* m, const zsme_settings* s, const double* p) {
    return new Oracle<MT, NT, zsme::Dual<1>>(m, s, p);
}
template <template <typename> class MT, template <typename> class NT>
OracleBase* make_counting(const zsme_mesh* m, const zsme_settings* s, const double* p) {
    return new Oracle<MT, NT, zsme::Counted>(m, s, p);
}

#define ORACLE_ENTRY(NS)                                                                   \
    Entry{#NS, &make_oracle<NS::Model, NS::Numerics>, &pointwise<NS::Model, NS::Numerics>,   \
          &flux_vjp<NS::Model, NS::Numerics>,                                              \
          NS::Model<double>::n_dof_q,                                                      \
          NS::Model<double>::n_dof_qaux, NS::Model<double>::n_parameters,                  \
          NS::Model<double>::dimension, &make_tlm<NS::Model, NS::Numerics>,                 \
          &make_counting<NS::Model, NS::Numerics>}

const Entry kEntries[] = {
    ORACLE_ENTRY(sme1d_l0_malpasset), ORACLE_ENTRY(sme2d_l0), ORACLE_ENTRY(sme2d_l1),
    ORACLE_ENTRY(sme2d_l2), ORACLE_ENTRY(sme2d_l4),
#ifdef ORACLE_WITH_REFERENCE_MODEL
    ORACLE_ENTRY(ref1d),
#endif
};

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

// Worker threads for the parallel loops (0 = all hardware threads).
int oracle_set_threads(int n) {
    g_threads = n > 0 ? n : (int)std::max(1u, std::thread::hardware_concurrency());
    return g_threads;
}

int oracle_model_info(const char* model, int* nq, int* na, int* np, int* dim) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) {
            *nq = e.nq; *na = e.na; *np = e.np; *dim = e.dim;
            return 0;
        }
    return fail(ZSME_ERR_MODEL, std::string("unknown model ") + model);
}

int oracle_create(const char* model, const zsme_mesh* mesh, const zsme_settings* s, const double* params,
                  void** out) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) {
            if (mesh->dim != e.dim) return fail(ZSME_ERR_ARG, "mesh dim != model dimension");
            *out = e.make(mesh, s, params);
            return 0;
        }
    return fail(ZSME_ERR_MODEL, std::string("unknown model ") + model);
}
int oracle_pointwise(const char* model, int fn, const double* qL, const double* qR, const double* aL,
                     const double* aR, const double* p, const double* n, double s, double* out) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) return e.pw(fn, qL, qR, aL, aR, p, n, s, out);
    return fail(-ZSME_ERR_MODEL, std::string("unknown model ") + model);
}
int oracle_flux_vjp(const char* model, const double* qL, const double* qR, const double* aL, const double* aR,
                    const double* p, const double* n, const double* w, double* g) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) return e.vjp(qL, qR, aL, aR, p, n, w, g);
    return fail(-ZSME_ERR_MODEL, std::string("unknown model ") + model);
}
// Tangent-linear instance: the same restatement on Dual<1> numbers.
int oracle_create_tlm(const char* model, const zsme_mesh* mesh, const zsme_settings* s, const double* params,
                      void** out) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) {
            if (mesh->dim != e.dim) return fail(ZSME_ERR_ARG, "mesh dim != model dimension");
            *out = e.make_tlm(mesh, s, params);
            return 0;
        }
    return fail(ZSME_ERR_MODEL, std::string("unknown model ") + model);
}
// Operation-counting instance (flopcount.h): the same restatement on
// Counted numbers; run it with one oracle thread.
int oracle_create_counting(const char* model, const zsme_mesh* mesh, const zsme_settings* s, const double* params,
                           void** out) {
    for (auto& e : kEntries)
        if (!std::strcmp(e.name, model)) {
            if (mesh->dim != e.dim) return fail(ZSME_ERR_ARG, "mesh dim != model dimension");
            *out = e.make_counting(mesh, s, params);
            return 0;
        }
    return fail(ZSME_ERR_MODEL, std::string("unknown model ") + model);
}
// out[phase * NOPS + op] (flopcount.h's Phase x Op), counted since the last reset
int oracle_flop_counts(long long* out) {
    for (int p = 0; p < zsme_flops::NPH; ++p)
        for (int o = 0; o < zsme_flops::NOPS; ++o) out[p * zsme_flops::NOPS + o] = zsme_flops::counts[p][o];
    return zsme_flops::NPH * zsme_flops::NOPS;
}
int oracle_flop_reset() {
    for (auto& r : zsme_flops::counts)
        for (auto& v : r) v = 0;
    return 0;
}
int oracle_set_tangent(void* h, const double* dq, const double* dp) { ((OracleBase*)h)->set_tangent(dq, dp); return 0; }
int oracle_get_tangent(void* h, double* dq) { ((OracleBase*)h)->get_tangent(dq); return 0; }
int oracle_destroy(void* h) { delete (OracleBase*)h; return 0; }
int oracle_set_state(void* h, const double* q, double t) { ((OracleBase*)h)->set_state(q, t); return 0; }
int oracle_get_state(void* h, double* q) { ((OracleBase*)h)->get_state(q); return 0; }
int oracle_get_aux(void* h, double* a) { ((OracleBase*)h)->get_aux(a); return 0; }
int oracle_rhs(void* h, double t, const double* x, double* f) { ((OracleBase*)h)->rhs(t, x, f); return 0; }
int oracle_gradient(void* h, const double* x, double* g) { ((OracleBase*)h)->gradient(x, g); return 0; }
int oracle_update_state(void* h) { ((OracleBase*)h)->update_state(); return 0; }
int oracle_source(void* h, double dt) { ((OracleBase*)h)->source(dt); return 0; }
int oracle_compute_dt(void* h, double* dt) { *dt = ((OracleBase*)h)->compute_dt(); return 0; }
int oracle_step(void* h, int n) { ((OracleBase*)h)->step(n, nullptr); return 0; }
int oracle_step_dt(void* h, int n, const double* dts) { ((OracleBase*)h)->step(n, dts); return 0; }
int oracle_get_time(void* h, double* t, double* dt) { ((OracleBase*)h)->get_time(t, dt); return 0; }
int oracle_set_params(void* h, const double* p) { ((OracleBase*)h)->set_params(p); return 0; }
int oracle_newton_unconverged(void* h) { return ((OracleBase*)h)->newton_unconverged(); }
int oracle_implicit_function(void* h, double t, const double* x, const double* xdot, double* f) {
    ((OracleBase*)h)->implicit_function(t, x, xdot, f);
    return 0;
}
int oracle_implicit_jacobian(void* h, double t, const double* x, double a, double* diag, double* faces) {
    ((OracleBase*)h)->implicit_jacobian(t, x, a, diag, faces);
    return 0;
}
int oracle_implicit_stats(void* h, int* out) { return ((OracleBase*)h)->implicit_stats(out); }
long long oracle_mood_cells(void* h) { return ((OracleBase*)h)->mood_cells(); }

}  // extern "C"
