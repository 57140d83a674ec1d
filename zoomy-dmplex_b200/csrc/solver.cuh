// Host side of one model's solver: device buffers, the CUDA stream, the
// captured CUDA graph of one time step, and the calls behind the C ABI.
// A solver advances one or several independent instances (an ensemble of
// meshes, concatenated cell- and face-wise); every kernel launch covers all
// instances.  Included once per model translation unit after the plugin.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "model_prelude.h"
#include "prepared_mesh.h"
#include "step_kernels.cuh"
#include "face_kernels.cuh"
#include "source_kernels.cuh"
#include "adjoint_kernels.cuh"
#include "imex_kernels.cuh"
#include "implicit_kernels.cuh"
#include "zsme.h"

namespace zsme {

#define ZSME_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return set_error(ZSME_ERR_CUDA, std::string(#call) + ": " +   \
                                                cudaGetErrorString(e_));                     \
    } while (0)

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t count) {
        if (p && n == count) return cudaSuccess;  // same size: keep the allocation
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (!count) return cudaSuccess;
        return cudaMalloc((void**)&p, count * sizeof(T));
    }
    cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(s);
    }
};

static inline int blocks_for(long long n, int b) { return (int)((n + b - 1) / b); }

template <template <typename> class MT, template <typename> class NT>
class Solver final : public SolverBase {
    using M = MT<double>;
    using N = NT<double>;
    static constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters, DIM = M::dimension;

    PreparedMesh pm_;
    zsme_settings st_{};
    int device_ = 0, n_inst_ = 1;
    LaunchConfig lc_{};
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    // mesh
    DevBuf<int> slot_nbr_, slot_meta_, slot_face_, order_, old_of_new_, face_L_, face_R_, face_bc_;
    DevBuf<int> new_of_old_, cells_tmp_;  // single-instance handles: caller -> device cell ids; zsme_*_cells staging
    DevBuf<int> cell_inst_, face_inst_;
    DevBuf<double> slot_dx_, slot_w_, vol_, rc_, fn_, farea_, fc_, fnr_;
    // state
    DevBuf<double> x_, w_, wl_, aux_, fs_, fb_, tmp_a_, tmp_b_, params_, dts_;
    double* fs_cur_ = nullptr;  // face states the prep and face kernels use: fs_, or a tape slot in a replay
    double* dec_cur_ = nullptr; // in a replay at order 2: the tape slot for the stage's reconstruction record
    // rows of one stage's reconstruction record (prep_tape_kernel): the gradient,
    // then alpha, dq and branch per face slot
    size_t dec_rows() const { return (size_t)NQ * DIM + 3 * (size_t)pm_.K; }
    DevBuf<double> xs_;  // MOOD: the state at the start of the step
    DevBuf<int> mood_list_;  // MOOD: the troubled cells of the step (count in iscal_[6])
    DevBuf<double> imex_g_[3], imex_s_[3], imex_y_[2];   // IMEX: stage right-hand sides, implicit derivatives, states
    static constexpr int kImpRestart = 30;   // GMRES restart length
    // fully implicit strategy (allocated with the handle when selected):
    // history X_n, X_{n-1}; residual F, trial residual, trial state, transport
    // RHS, Krylov basis [31][NQ C], work, Newton update, preconditioned
    // residual at zero, restart residual; clamped state and its aux; the
    // assembled diagonal blocks, their LU factors and pivots; the face blocks
    DevBuf<double> imp_xn_, imp_xnm1_, imp_F_, imp_Ft_, imp_xt_, imp_R_, imp_V_, imp_w_, imp_d_, imp_r0_, imp_r_;
    DevBuf<double> imp_xl_, imp_al_, imp_pd_, imp_lu_, imp_fj_, imp_part_, imp_red_;
    // device scalars of the step: [0] t_{n+1}, [1] |X|, [2..5] BDF c0, c1, c2, h,
    // [6] v.v, [7] differencing parameter, [8] w.w, [9] X.X
    DevBuf<double> imp_scal_;
    DevBuf<int> imp_piv_;
    cudaGraphExec_t imp_graph_[kImpRestart] = {};   // Arnoldi step j, captured on first use
    bool imp_have_prev_ = false;   // a previous implicit step exists: BDF2
    double imp_h_prev_ = 0.0;
    int imp_stats_[4] = {0, 0, 0, 0};   // last step: Newton iterations, GMRES iterations, halvings, converged

    // per instance: t, dt_cfl, dt_step, dt_aux ; active ; ratio
    DevBuf<double> t_, dt_cfl_, dt_step_, dt_aux_;
    DevBuf<int> active_, iscal_;  // iscal_: [0] step_idx, [1..4] diag, [5] deferred finalize cells, [6] MOOD cells
    DevBuf<int> fin_list_;        // [C] cells deferred to the generic Newton path
    // tiles of the fused face + gather kernel (LaunchConfig::tile_faces > 0)
    DevBuf<int> tile_cell_off_, tile_face_off_, tile_in_off_, tile_in_faces_, tile_ord_lf_;
    int tile_n_ = 0, tile_stride_ = 0, tile_built_ = 0;  // tile_built_: the tile_faces they were built for
    bool ready_ = false;          // init done: mesh on the device
    bool lean_ok_ = false;        // 32-bit element offsets cover every array prep_lean_kernel indexes
    DerivSpecs deriv_{};          // derivative aux slots refreshed at every state update (n = 0: none)
    int sm_count_ = 148;
    DevBuf<unsigned long long> ratio_;
    // discrete adjoint (allocated by the first zsme_adjoint call)
    DevBuf<double> adj_ck_x_, adj_ck_a_, adj_tape_, adj_lam0_, adj_lam1_, adj_lam2_, adj_own_w_, adj_own_wl_;
    DevBuf<double> adj_out_w_, adj_out_wl_, adj_gfs_, adj_lp_cell_, adj_lp_, adj_wl_, adj_oval_, adj_oseed_, adj_dts_;
    DevBuf<int> adj_ocell_, adj_ocomp_, adj_first_, adj_segn0_all_, adj_seg_n0_;
    DevBuf<double> adj_th_, adj_seg_dt_, adj_seg_t_;
    size_t adj_tstride_ = 0;
    // two tape buffers when the replay of one checkpoint segment overlaps the
    // reverse sweep of the next (side stream); adj_par_ selects the buffer the
    // enqueued replay / reverse launches use, adj_aux_cur_ the aux array the
    // reverse launches read (the live aux, or its snapshot at the end of the
    // segment's replay)
    DevBuf<double> adj_aux_snap_;
    cudaStream_t adj_side_ = nullptr;
    int adj_par_ = 0, adj_tape_steps_ = 0;
    const double* adj_aux_cur_ = nullptr;
    bool adj_overlapped_ = false;  // the last zsme_adjoint overlapped its replays with the reverse sweep
    double adj_phase_ms_[3] = {0, 0, 0};  // last zsme_adjoint: forward pass, replays, reverse sweep
    MeshDev md_{};
    Opts opts_{};
    // per-kernel CUDA-event timing (zsme_set_profiling)
    bool profiling_ = false;
    bool x_clamped_ = true;  // x_ equals update_variables(x_)
    std::vector<cudaEvent_t> ev_pool_;
    // asynchronous state I/O (zsme_set_state_async / zsme_get_state_async)
    cudaStream_t h2d_ = nullptr, d2h_ = nullptr;
    DevBuf<double> in_stage_[2], out_stage_[2];
    cudaEvent_t ev_h2d_[2] = {}, ev_in_used_[2] = {}, ev_out_[2] = {}, ev_d2h_[2] = {};
    int in_k_ = 0, out_k_ = 0, last_d2h_ = 0;
    std::vector<int> ev_kind_;
    size_t ev_used_ = 0;
    double prof_ms_[ZSME_KERNEL_KINDS] = {0};
    int64_t prof_n_[ZSME_KERNEL_KINDS] = {0};

  public:
    ~Solver() override {
        if (graph_) cudaGraphExecDestroy(graph_);
        imp_drop_graphs();
        for (auto e : ev_pool_) cudaEventDestroy(e);
        if (h2d_) {
            cudaStreamSynchronize(h2d_);
            cudaStreamSynchronize(d2h_);
            for (int j = 0; j < 2; ++j)
                for (cudaEvent_t e : {ev_h2d_[j], ev_in_used_[j], ev_out_[j], ev_d2h_[j]}) cudaEventDestroy(e);
            cudaStreamDestroy(h2d_);
            cudaStreamDestroy(d2h_);
        }
        if (adj_side_) cudaStreamDestroy(adj_side_);
        if (stream_) cudaStreamDestroy(stream_);
    }

    int n_dof_q() const override { return NQ; }
    int n_dof_qaux() const override { return NA; }
    int n_instances() const override { return n_inst_; }
    int device() const override { return device_; }

    // ------------------------------------------------------- profiling
    void mark(int kind, bool start) {
        if (!profiling_) return;
        if (start) {
            if (ev_used_ + 2 > ev_pool_.size()) {
                for (int i = 0; i < 64; ++i) {
                    cudaEvent_t e;
                    cudaEventCreate(&e);
                    ev_pool_.push_back(e);
                }
                ev_kind_.resize(ev_pool_.size() / 2);
            }
            ev_kind_[ev_used_ / 2] = kind;
        }
        cudaEventRecord(ev_pool_[ev_used_], stream_);
        ev_used_++;
    }
    int collect_profile() {
        if (!profiling_ || !ev_used_) return ZSME_OK;
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        for (size_t i = 0; i + 1 < ev_used_; i += 2) {
            float ms = 0.f;
            ZSME_CUDA(cudaEventElapsedTime(&ms, ev_pool_[i], ev_pool_[i + 1]));
            prof_ms_[ev_kind_[i / 2]] += ms;
            prof_n_[ev_kind_[i / 2]] += 1;
        }
        ev_used_ = 0;
        return ZSME_OK;
    }
    int set_profiling(int on) override {
        profiling_ = on != 0;
        ev_used_ = 0;
        for (int k = 0; k < ZSME_KERNEL_KINDS; ++k) { prof_ms_[k] = 0; prof_n_[k] = 0; }
        return ZSME_OK;
    }
    int read_profile(double* ms, int64_t* n) override {
        for (int k = 0; k < ZSME_KERNEL_KINDS; ++k) {
            if (ms) ms[k] = prof_ms_[k];
            if (n) n[k] = prof_n_[k];
        }
        return ZSME_OK;
    }

    // ------------------------------------------------------- set-up
    int set_launch(const LaunchConfig& lc) override {
        for (int b : {lc.prep, lc.face, lc.gather, lc.finalize})
            if (b < 32 || b > 128 || b % 32) return set_error(ZSME_ERR_ARG, "block sizes must be 32, 64, 96 or 128");
        if (lc.prep_occ < 1 || lc.prep_occ > 8 || lc.prep_occ == 5 || lc.prep_occ == 7)
            return set_error(ZSME_ERR_ARG, "prep occupancy cap must be 1, 2, 3, 4, 6 or 8 blocks per SM");
        if (lc.face_occ < 1 || lc.face_occ > 4 || lc.finalize_occ < 1 || lc.finalize_occ > 4)
            return set_error(ZSME_ERR_ARG, "face and finalize occupancy caps must be 1..4 blocks per SM");
        if (lc.fuse_final < 0 || lc.fuse_final > 1) return set_error(ZSME_ERR_ARG, "fuse_final must be 0 or 1");
        if (lc.prep_lean < 0 || lc.prep_lean > 4)
            return set_error(ZSME_ERR_ARG, "prep_lean must be 0 (plain), 1 (lean) or 2..4 (lean, threads per cell)");
        if (lc.tile_faces != 0 && (lc.tile_faces < 64 || lc.tile_faces > 1024))
            return set_error(ZSME_ERR_ARG, "tile_faces must be 0 (separate face and gather kernels) or 64..1024");
        if ((size_t)lc.tile_faces * 3 * NQ * sizeof(double) > kMaxTileSmem)
            return set_error(ZSME_ERR_ARG, "tile_faces too large for this model's shared-memory rows (at most " +
                                               std::to_string(kMaxTileSmem / (3 * NQ * sizeof(double))) + ")");
        lc_ = lc;
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        imp_drop_graphs();
        if (ready_) return ensure_tiles();
        return ZSME_OK;
    }
    // Shared memory of one tile: 3 NQ rows of the tile's faces.
    static constexpr size_t kMaxTileSmem = 200 * 1024;
    // (Re)builds the tiles for lc_.tile_faces; outside any stream capture
    // (set-up and zsme_set_launch only).
    int ensure_tiles() {
        if (lc_.tile_faces <= 0 || tile_built_ == lc_.tile_faces) return ZSME_OK;
        FaceTiles t;
        int rc = build_tiles(pm_, lc_.tile_faces, t);
        if (rc) return rc;
        ZSME_CUDA(tile_cell_off_.upload(t.cell_off, stream_));
        ZSME_CUDA(tile_face_off_.upload(t.face_off, stream_));
        ZSME_CUDA(tile_in_off_.upload(t.in_off, stream_));
        if (t.in_faces.empty()) t.in_faces.push_back(0);
        ZSME_CUDA(tile_in_faces_.upload(t.in_faces, stream_));
        ZSME_CUDA(tile_ord_lf_.upload(t.ord_lf, stream_));
        tile_n_ = t.n;
        tile_stride_ = t.max_faces;
        const int smem = (int)((size_t)tile_stride_ * 3 * NQ * sizeof(double));
        ZSME_CUDA(cudaFuncSetAttribute(flux_tile_kernel<M, N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ZSME_CUDA(cudaFuncSetAttribute(flux_tile_kernel<M, N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ZSME_CUDA(cudaFuncSetAttribute(flux_tile_kernel<M, N, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ZSME_CUDA(cudaFuncSetAttribute(flux_tile_kernel<M, N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        tile_built_ = lc_.tile_faces;
        return ZSME_OK;
    }
    LaunchConfig launch() const override { return lc_; }

    int init(PreparedMesh&& pm, const zsme_settings& st, const double* params, int device) override {
        pm_ = std::move(pm);
        st_ = st;
        device_ = device;
        n_inst_ = pm_.n_inst;
        if (pm_.dim != DIM) return set_error(ZSME_ERR_ARG, "mesh dimension does not match the model");
        if (st_.reconstruction_order >= 2 && st_.ssp_stages < 2)
            return set_error(ZSME_ERR_ARG, "ssp_stages must be >= 2");
        if (st_.time_integration != ZSME_TIME_SPLITTING && st_.time_integration != ZSME_TIME_IMEX &&
            st_.time_integration != ZSME_TIME_IMPLICIT)
            return set_error(ZSME_ERR_ARG,
                             "time_integration must be ZSME_TIME_SPLITTING, ZSME_TIME_IMEX or ZSME_TIME_IMPLICIT");
        if (st_.time_integration == ZSME_TIME_IMPLICIT &&
            (n_inst_ != 1 || st_.positivity == ZSME_POSITIVITY_MOOD))
            return set_error(ZSME_ERR_ARG, "the implicit strategy needs a single-instance handle and positivity "
                                           "other than \"mood\"");
        if (st_.positivity != ZSME_POSITIVITY_NONE && (NQ < 3 || !(st_.wet_dry_eps >= 0)))
            return set_error(ZSME_ERR_ARG, "positivity variants need a [b, h, momentum...] model and wet_dry_eps >= 0");
        // Zhang-Shu positivity holds for CFL <= 1/6 at order 2 (MUSCLSolver.hpp:33-38)
        if (st_.reconstruction_order >= 2 && st_.positivity == ZSME_POSITIVITY_ZHANG_SHU && st_.cfl > 1.0 / 6.0)
            st_.cfl = 1.0 / 6.0;
        ZSME_CUDA(cudaSetDevice(device_));
        ZSME_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        ZSME_CUDA(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device_));
        LaunchConfig lc{128, 128, 128, 128};
        // fused face + gather tiles of up to 256 faces, smaller while the mesh
        // would give fewer than three tiles per SM
        int tf = std::min(256, (int)(kMaxTileSmem / (3 * NQ * sizeof(double))));
        while (tf > 64 && pm_.F / tf < 3 * sm_count_) tf /= 2;
        lc.tile_faces = tf;
        if (st_.block_size > 0) lc.prep = lc.face = lc.gather = st_.block_size;
        int rc = set_launch(lc);
        if (rc) return rc;
        const int C = pm_.C, F = pm_.F;
        ZSME_CUDA(slot_nbr_.upload(pm_.slot_nbr, stream_));
        ZSME_CUDA(slot_meta_.upload(pm_.slot_meta, stream_));
        ZSME_CUDA(slot_face_.upload(pm_.slot_face, stream_));
        ZSME_CUDA(order_.upload(pm_.order, stream_));
        ZSME_CUDA(old_of_new_.upload(pm_.old_of_new, stream_));
        if (n_inst_ == 1) ZSME_CUDA(new_of_old_.upload(pm_.new_of_old, stream_));
        ZSME_CUDA(slot_dx_.upload(pm_.slot_dx, stream_));
        ZSME_CUDA(slot_w_.upload(pm_.slot_w, stream_));
        ZSME_CUDA(vol_.upload(pm_.vol, stream_));
        ZSME_CUDA(rc_.upload(pm_.rc, stream_));
        ZSME_CUDA(fn_.upload(pm_.fn, stream_));
        ZSME_CUDA(farea_.upload(pm_.farea, stream_));
        ZSME_CUDA(fc_.upload(pm_.fc, stream_));
        ZSME_CUDA(fnr_.upload(pm_.fnr, stream_));
        ZSME_CUDA(face_L_.upload(pm_.face_L, stream_));
        ZSME_CUDA(face_R_.upload(pm_.face_R, stream_));
        ZSME_CUDA(face_bc_.upload(pm_.face_bc, stream_));
        if (n_inst_ > 1) {
            ZSME_CUDA(cell_inst_.upload(pm_.cell_inst, stream_));
            ZSME_CUDA(face_inst_.upload(pm_.face_inst, stream_));
        }
        md_ = MeshDev{C, pm_.K, slot_nbr_.p, slot_meta_.p, slot_face_.p, slot_dx_.p, slot_w_.p, vol_.p,
                      rc_.p, order_.p, fn_.p, farea_.p, fc_.p, fnr_.p, F, face_L_.p, face_R_.p,
                      face_bc_.p, cell_inst_.p, face_inst_.p, NP};
        opts_ = Opts{st_.reconstruction_order, st_.limiter, st_.gradient, st_.ssp_stages, st_.source};
        ZSME_CUDA(x_.alloc((size_t)NQ * C));
        ZSME_CUDA(w_.alloc((size_t)NQ * C));
        ZSME_CUDA(wl_.alloc((size_t)NQ * C));
        ZSME_CUDA(aux_.alloc((size_t)NA * C));
        if (st_.time_integration == ZSME_TIME_IMEX) {
            for (int j = 0; j < 3; ++j) {
                ZSME_CUDA(imex_g_[j].alloc((size_t)NQ * C));
                ZSME_CUDA(imex_s_[j].alloc((size_t)NQ * C));
            }
            for (int j = 0; j < 2; ++j) ZSME_CUDA(imex_y_[j].alloc((size_t)NQ * C));
        }
        if (st_.time_integration == ZSME_TIME_IMPLICIT) {
            const size_t n = (size_t)NQ * C;
            for (auto* b : {&imp_xn_, &imp_xnm1_, &imp_F_, &imp_Ft_, &imp_xt_, &imp_R_, &imp_w_, &imp_d_, &imp_r0_,
                            &imp_r_, &imp_xl_})
                ZSME_CUDA(b->alloc(n));
            ZSME_CUDA(imp_V_.alloc((size_t)(kImpRestart + 1) * n));
            ZSME_CUDA(imp_al_.alloc((size_t)NA * C + 1));
            ZSME_CUDA(imp_pd_.alloc((size_t)NQ * NQ * C));
            ZSME_CUDA(imp_lu_.alloc((size_t)NQ * NQ * C));
            ZSME_CUDA(imp_piv_.alloc((size_t)NQ * C));
            ZSME_CUDA(imp_fj_.alloc((size_t)4 * NQ * NQ * F));
            ZSME_CUDA(imp_part_.alloc((size_t)(kImpRestart + 1) * imp_dot_blocks()));
            ZSME_CUDA(imp_red_.alloc((size_t)kImpRestart + 8));
            ZSME_CUDA(imp_scal_.alloc(16));
        }
        if (st_.positivity == ZSME_POSITIVITY_MOOD) {
            ZSME_CUDA(xs_.alloc((size_t)NQ * C));
            ZSME_CUDA(mood_list_.alloc((size_t)C));
        }
        ZSME_CUDA(fs_.alloc((size_t)2 * NQ * F));
        fs_cur_ = fs_.p;
        ZSME_CUDA(fb_.alloc((size_t)3 * NQ * F));
        // staging for state (NQ per cell) and aux (NA per cell) conversions
        ZSME_CUDA(tmp_a_.alloc((size_t)std::max(NQ, NA) * C));
        ZSME_CUDA(tmp_b_.alloc((size_t)std::max(NQ, NA) * C));
        ZSME_CUDA(cudaMemsetAsync(x_.p, 0, x_.n * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(aux_.p, 0, aux_.n * sizeof(double), stream_));
        for (auto* b : {&t_, &dt_cfl_, &dt_step_, &dt_aux_}) {
            ZSME_CUDA(b->alloc(n_inst_));
            ZSME_CUDA(cudaMemsetAsync(b->p, 0, n_inst_ * sizeof(double), stream_));
        }
        ZSME_CUDA(fin_list_.alloc((size_t)C));
        ZSME_CUDA(active_.alloc(n_inst_));
        ZSME_CUDA(cudaMemsetAsync(active_.p, 0, n_inst_ * sizeof(int), stream_));
        ZSME_CUDA(iscal_.alloc(8));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, 8 * sizeof(int), stream_));
        ZSME_CUDA(ratio_.alloc(n_inst_));
        std::vector<unsigned long long> none(n_inst_, ZSME_RATIO_NONE);
        ZSME_CUDA(cudaMemcpyAsync(ratio_.p, none.data(), n_inst_ * sizeof(unsigned long long),
                                  cudaMemcpyHostToDevice, stream_));
        std::vector<double> pv((size_t)NP * n_inst_);
        auto dp = M::default_parameters();
        for (int i = 0; i < n_inst_; ++i)
            for (int k = 0; k < NP; ++k) pv[(size_t)i * NP + k] = params ? params[(size_t)i * NP + k] : dp[k];
        ZSME_CUDA(params_.upload(pv, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        lean_ok_ = 2LL * NQ * F < 0x7fffffffLL && (long long)NQ * C < 0x7fffffffLL &&
                   (long long)pm_.K * 2 * C < 0x7fffffffLL;
        if (st_.refresh_derivative_aux) {
            int rc2 = record_derivative_aux();
            if (rc2) return rc2;
        }
        ready_ = true;
        return ensure_tiles();
    }

    // The plugin's field-level update_aux_variables, called once on the host
    // with one stand-in pointer per field: each compute_derivative request it
    // makes is recorded as (aux slot, state variable, axis, order) for
    // derivative_aux_kernel.  Plugins without the overload record nothing.
    struct DerivRecorder {
        const double* qf;
        const double* af;
        DerivSpecs* ds;
        bool bad;
    };
    static void record_request(const ZoomyMesh& mesh, double* result, const double* source, int dx, int dy, int dz) {
        auto* r = static_cast<DerivRecorder*>(mesh.ctx);
        const long k = result - r->af, i = source - r->qf;
        const int total = dx + dy + dz;
        if (k < 0 || k >= NA || i < 0 || i >= NQ || total > 1 || r->ds->n >= 8) {
            r->bad = true;
            return;
        }
        const int e = r->ds->n++;
        r->ds->aux[e] = (int)k;
        r->ds->comp[e] = (int)i;
        r->ds->axis[e] = dx == 1 ? 0 : (dy == 1 ? 1 : 2);
        r->ds->order[e] = total;
    }
    int record_derivative_aux() {
        deriv_ = DerivSpecs{};
        if constexpr (HasFieldAuxUpdate<M>::value) {
            double qf[NQ] = {}, af[NA] = {};
            double* Qp[NQ];
            double* Ap[NA];
            for (int i = 0; i < NQ; ++i) Qp[i] = &qf[i];
            for (int k = 0; k < NA; ++k) Ap[k] = &af[k];
            DerivRecorder rec{qf, af, &deriv_, false};
            const ZoomyMesh mesh{&Solver::record_request, &rec};
            M::update_aux_variables(Qp, Ap, 0.0, mesh);
            if (rec.bad)
                return set_error(ZSME_ERR_MODEL, "the plugin's field-level update_aux_variables asks for a derivative "
                                                 "this solver does not provide (state variable to aux slot, first "
                                                 "order, at most 8)");
        }
        return ZSME_OK;
    }
    // RefreshDerivativeAux of state xs into aux_ (no-op without derivative slots)
    void launch_derivative_aux(const double* xs, const int* active) {
        if (!deriv_.n) return;
        derivative_aux_kernel<M><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, deriv_, 0, pm_.C, xs, aux_.p,
                                                                             active);
    }

    StepDev step_dev(const double* dts) {
        return StepDev{t_.p, dt_cfl_.p, dt_step_.p, active_.p, ratio_.p, dts, iscal_.p + 0, n_inst_,
                       st_.t_end, st_.cfl, M::dt_max, iscal_.p + 1, fin_list_.p, iscal_.p + 5};
    }

    int set_params(const double* params) override {
        ZSME_CUDA(cudaMemcpyAsync(params_.p, params, (size_t)NP * n_inst_ * sizeof(double), cudaMemcpyHostToDevice,
                                  stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    int check_inst(int i) const {
        if (i < 0 || i >= n_inst_) return set_error(ZSME_ERR_ARG, "instance index out of range");
        return ZSME_OK;
    }

    // ---------------------------------------------------------- state I/O
    int set_state(int inst, const double* q, double t, bool device) override {
        int rc = check_inst(inst);
        if (rc) return rc;
        const int c0 = pm_.inst_cell_off[inst], cn = pm_.inst_cell_off[inst + 1] - c0;
        const double* src = q;
        if (!device) {
            ZSME_CUDA(cudaMemcpyAsync(tmp_a_.p, q, (size_t)NQ * cn * sizeof(double), cudaMemcpyHostToDevice, stream_));
            src = tmp_a_.p;
        }
        aos_to_soa_kernel<<<blocks_for(cn, 128), 128, 0, stream_>>>(src, x_.p, old_of_new_.p, c0, cn, pm_.C, NQ);
        ZSME_CUDA(cudaGetLastError());
        set_time_kernel<<<1, 1, 0, stream_>>>(t_.p + inst, t);
        rc = enqueue_loaded(inst, c0, cn);
        if (rc) return rc;
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }
    // After a state (and its time) is in place: aux reset, constraints, then
    // dt_start = max(ComputeTimeStep, min_dt) (MUSCLSolver.hpp:51-54, 103).
    int enqueue_loaded(int inst, int c0, int cn) {
        imp_have_prev_ = false;   // the implicit strategy restarts at BDF order 1
        for (int k = 0; k < NA; ++k)
            ZSME_CUDA(cudaMemsetAsync(aux_.p + (size_t)k * pm_.C + c0, 0, cn * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(active_.p + inst, 0, sizeof(int), stream_));
        if (inst == 0) ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, 8 * sizeof(int), stream_));
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        launch_derivative_aux(x_.p, nullptr);      // PostStep's UpdateState: the derivative aux first
        finalize_range(c0, cn, sd, nullptr, FIN_POST | FIN_WRITE | FIN_DT);
        ZSME_CUDA(cudaGetLastError());
        end_step_kernel<<<1, 32, 0, stream_>>>(step_dev(nullptr), inst, 1, 0, st_.min_dt, nullptr);
        ZSME_CUDA(cudaGetLastError());
        x_clamped_ = true;
        return ZSME_OK;
    }

    // ------------------------------------------------ cell subsets (halo exchange)
    int cells_io(int n, const int* cells, double* q_get, const double* q_set, bool device) {
        const int C = pm_.C;
        if (n < 0 || n > C) return set_error(ZSME_ERR_ARG, "cell count out of range");
        if (n == 0) return ZSME_OK;
        const int* dc = cells;
        double* dq = q_get ? q_get : const_cast<double*>(q_set);
        if (!device) {
            for (int e = 0; e < n; ++e)
                if (cells[e] < 0 || cells[e] >= C) return set_error(ZSME_ERR_ARG, "cell id out of range");
            ZSME_CUDA(cells_tmp_.alloc((size_t)C));
            ZSME_CUDA(cudaMemcpyAsync(cells_tmp_.p, cells, n * sizeof(int), cudaMemcpyHostToDevice, stream_));
            dc = cells_tmp_.p;
            dq = tmp_a_.p;
            if (q_set)
                ZSME_CUDA(cudaMemcpyAsync(tmp_a_.p, q_set, (size_t)n * NQ * sizeof(double), cudaMemcpyHostToDevice,
                                          stream_));
        }
        if (q_get) {
            get_cells_kernel<<<blocks_for(n, 128), 128, 0, stream_>>>(x_.p, C, NQ, new_of_old_.p, dc, n, dq);
            ZSME_CUDA(cudaGetLastError());
            if (!device) {
                ZSME_CUDA(cudaMemcpyAsync(q_get, tmp_a_.p, (size_t)n * NQ * sizeof(double), cudaMemcpyDeviceToHost,
                                          stream_));
                ZSME_CUDA(cudaStreamSynchronize(stream_));
            }
        } else {
            set_cells_kernel<M><<<blocks_for(n, 128), 128, 0, stream_>>>(x_.p, aux_.p, C, new_of_old_.p, dc, n, dq,
                                                                        params_.p);
            ZSME_CUDA(cudaGetLastError());
            if (!device) ZSME_CUDA(cudaStreamSynchronize(stream_));
        }
        return ZSME_OK;
    }
    int get_cells(int n, const int* cells, double* q, bool device) override {
        return cells_io(n, cells, q, nullptr, device);
    }
    int set_cells(int n, const int* cells, const double* q, bool device) override {
        return cells_io(n, cells, nullptr, q, device);
    }

    // ------------------------------------------------ asynchronous state I/O
    // Host <-> device state copies on two copy streams (one per direction)
    // through double-buffered device staging, ordered against the handle's
    // stream by events: a copy in one direction, the other direction's copy
    // and the steps in between can all be in flight at once.
    int async_setup() {
        if (h2d_) return ZSME_OK;
        const size_t n = (size_t)NQ * pm_.C;
        for (int j = 0; j < 2; ++j) {
            ZSME_CUDA(in_stage_[j].alloc(n));
            ZSME_CUDA(out_stage_[j].alloc(n));
            for (cudaEvent_t* e : {&ev_h2d_[j], &ev_in_used_[j], &ev_out_[j], &ev_d2h_[j]})
                ZSME_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        }
        ZSME_CUDA(cudaStreamCreateWithFlags(&d2h_, cudaStreamNonBlocking));
        ZSME_CUDA(cudaStreamCreateWithFlags(&h2d_, cudaStreamNonBlocking));
        return ZSME_OK;
    }
    int set_state_async(const double* q, double t) override {
        int rc = async_setup();
        if (rc) return rc;
        const int j = in_k_;
        in_k_ ^= 1;
        const int C = pm_.C;
        // staging buffer j is free once the conversion of two calls ago has read it
        ZSME_CUDA(cudaStreamWaitEvent(h2d_, ev_in_used_[j], 0));
        ZSME_CUDA(cudaMemcpyAsync(in_stage_[j].p, q, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, h2d_));
        ZSME_CUDA(cudaEventRecord(ev_h2d_[j], h2d_));
        ZSME_CUDA(cudaStreamWaitEvent(stream_, ev_h2d_[j], 0));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(in_stage_[j].p, x_.p, old_of_new_.p, 0, C, C, NQ);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaEventRecord(ev_in_used_[j], stream_));
        set_time_kernel<<<1, 1, 0, stream_>>>(t_.p, t);
        return enqueue_loaded(0, 0, C);
    }
    int get_state_async(double* q) override {
        int rc = async_setup();
        if (rc) return rc;
        const int j = out_k_;
        out_k_ ^= 1;
        const int C = pm_.C;
        // staging buffer j is free once its copy of two calls ago has left the device
        ZSME_CUDA(cudaStreamWaitEvent(stream_, ev_d2h_[j], 0));
        soa_to_aos_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(x_.p, out_stage_[j].p, old_of_new_.p, 0, C, C, NQ);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaEventRecord(ev_out_[j], stream_));
        ZSME_CUDA(cudaStreamWaitEvent(d2h_, ev_out_[j], 0));
        ZSME_CUDA(cudaMemcpyAsync(q, out_stage_[j].p, (size_t)NQ * C * sizeof(double), cudaMemcpyDeviceToHost, d2h_));
        ZSME_CUDA(cudaEventRecord(ev_d2h_[j], d2h_));
        last_d2h_ = j;
        return ZSME_OK;
    }
    int stream_wait_copies() override {
        if (!h2d_) return ZSME_OK;
        ZSME_CUDA(cudaStreamWaitEvent(stream_, ev_d2h_[last_d2h_], 0));
        ZSME_CUDA(cudaStreamWaitEvent(stream_, ev_h2d_[in_k_ ^ 1], 0));
        return ZSME_OK;
    }

    int get_soa(int inst, const double* soa, int nv, double* out, bool device) {
        const int c0 = pm_.inst_cell_off[inst], cn = pm_.inst_cell_off[inst + 1] - c0;
        double* dst = device ? out : tmp_b_.p;
        soa_to_aos_kernel<<<blocks_for(cn, 128), 128, 0, stream_>>>(soa, dst, old_of_new_.p, c0, cn, pm_.C, nv);
        ZSME_CUDA(cudaGetLastError());
        if (!device)
            ZSME_CUDA(cudaMemcpyAsync(out, tmp_b_.p, (size_t)nv * cn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }
    int get_state(int inst, double* q, bool device) override {
        int rc = check_inst(inst);
        return rc ? rc : get_soa(inst, x_.p, NQ, q, device);
    }
    int get_aux(int inst, double* a) override {
        int rc = check_inst(inst);
        return rc ? rc : get_soa(inst, aux_.p, NA, a, false);
    }

    // ---------------------------------------------------------- pieces
    // w: stage state, wl: its clamped copy (the same array where w is already clamped)
    void launch_prep(const double* w, const double* wl, const int* active) {
        mark(ZSME_KERNEL_PREP, true);
        const int gb = blocks_for(pm_.C, lc_.prep);
        if (dec_cur_ && st_.positivity == ZSME_POSITIVITY_NONE) {   // adjoint replay: record the reconstruction
            if (pm_.K == 3)
                prep_tape_kernel<M, 3><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl,
                                                                                   params_.p, fs_cur_, dec_cur_,
                                                                                   active);
            else
                prep_tape_kernel<M, 4><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl,
                                                                                   params_.p, fs_cur_, dec_cur_,
                                                                                   active);
            mark(ZSME_KERNEL_PREP, false);
            return;
        }
        if (st_.positivity != ZSME_POSITIVITY_NONE && st_.reconstruction_order >= 2) {
            switch (lc_.prep_occ) {
#define ZSME_PREPWB(OCC)                                                                                        \
    case OCC:                                                                                                   \
        if (pm_.K == 3)                                                                                         \
            prep_wb_kernel<M, 3, OCC><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, st_.positivity, st_.wet_dry_eps, \
                                                                    0, pm_.C, w, wl, params_.p, fs_cur_, active); \
        else                                                                                                    \
            prep_wb_kernel<M, 4, OCC><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, st_.positivity, st_.wet_dry_eps, \
                                                                    0, pm_.C, w, wl, params_.p, fs_cur_, active); \
        break;
                ZSME_PREPWB(2) ZSME_PREPWB(3) ZSME_PREPWB(4) ZSME_PREPWB(6) ZSME_PREPWB(8)
                default: ZSME_PREPWB(1)
#undef ZSME_PREPWB
            }
            mark(ZSME_KERNEL_PREP, false);
            return;
        }
        if (lc_.prep_lean >= 2 && st_.reconstruction_order >= 2 && lean_ok_) {
            switch (lc_.prep_lean) {
                case 2: launch_prep_split<2>(w, wl, active); break;
                case 3: launch_prep_split<3>(w, wl, active); break;
                default: launch_prep_split<4>(w, wl, active); break;
            }
            mark(ZSME_KERNEL_PREP, false);
            return;
        }
        if (lc_.prep_lean && st_.reconstruction_order >= 2 && lean_ok_) {
            switch (lc_.prep_occ) {
#define ZSME_PREPL(OCC)                                                                                         \
    case OCC:                                                                                                   \
        if (pm_.K == 3)                                                                                         \
            prep_lean_kernel<M, OCC, 3><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, params_.p,   \
                                                                      fs_cur_, active);                         \
        else                                                                                                    \
            prep_lean_kernel<M, OCC, 4><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, params_.p,   \
                                                                      fs_cur_, active);                         \
        break;
                ZSME_PREPL(2) ZSME_PREPL(3) ZSME_PREPL(4) ZSME_PREPL(6) ZSME_PREPL(8)
                default: ZSME_PREPL(1)
#undef ZSME_PREPL
            }
            mark(ZSME_KERNEL_PREP, false);
            return;
        }
        switch (lc_.prep_occ) {
#define ZSME_PREP(OCC)                                                                                          \
    case OCC:                                                                                                   \
        if (pm_.K == 3)                                                                                         \
            prep_kernel<M, OCC, 3><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, aux_.p, params_.p,\
                                                                 fs_cur_, active);                              \
        else                                                                                                    \
            prep_kernel<M, OCC, 4><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, aux_.p, params_.p,\
                                                                 fs_cur_, active);                              \
        break;
            ZSME_PREP(2) ZSME_PREP(3) ZSME_PREP(4) ZSME_PREP(6) ZSME_PREP(8)
            default: ZSME_PREP(1)
#undef ZSME_PREP
        }
        mark(ZSME_KERNEL_PREP, false);
    }
    // prep_lean_kernel's face states, P threads per cell (prep_split_kernel)
    template <int P>
    void launch_prep_split(const double* w, const double* wl, const int* active) {
        const int gb = blocks_for(pm_.C, SplitShape<P>::CB);
        constexpr int T = SplitShape<P>::threads;
        switch (lc_.prep_occ) {
#define ZSME_PREPS(OCC)                                                                                         \
    case OCC:                                                                                                   \
        if (pm_.K == 3)                                                                                         \
            prep_split_kernel<M, OCC, 3, P><<<gb, T, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, params_.p,      \
                                                                   fs_cur_, active);                            \
        else                                                                                                    \
            prep_split_kernel<M, OCC, 4, P><<<gb, T, 0, stream_>>>(md_, opts_, 0, pm_.C, w, wl, params_.p,      \
                                                                   fs_cur_, active);                            \
        break;
            ZSME_PREPS(4) ZSME_PREPS(6) ZSME_PREPS(8)
            default: ZSME_PREPS(1)
#undef ZSME_PREPS
        }
    }
    // face_only: the face kernel alone (split path), its gather left to the
    // finalize kernel (fused_final_stage)
    void launch_flux(int mode, double t_host, const double* t_dev, double frac, const double* x_in, double* x_out,
                     double* base, const double* dt, const int* active, double* xl_out = nullptr,
                     bool face_only = false) {
        if (lc_.tile_faces > 0) {   // fused face + gather over tiles
            mark(ZSME_KERNEL_FLUX, true);
            const TilesDev tl{tile_cell_off_.p, tile_face_off_.p, tile_in_off_.p, tile_in_faces_.p, tile_ord_lf_.p,
                              tile_stride_};
            const size_t smem = (size_t)tile_stride_ * 3 * NQ * sizeof(double);
            switch (lc_.face_occ) {
#define ZSME_TILE(OCC)                                                                                        \
    case OCC:                                                                                                 \
        flux_tile_kernel<M, N, OCC><<<tile_n_, lc_.face, smem, stream_>>>(md_, opts_, tl, fs_cur_, aux_.p,      \
                                                                       params_.p, t_host, t_dev, frac, dt,     \
                                                                       active, mode, x_in, x_out, base,        \
                                                                       xl_out);                                \
        break;
                ZSME_TILE(2) ZSME_TILE(3) ZSME_TILE(4)
                default: ZSME_TILE(1)
#undef ZSME_TILE
            }
            mark(ZSME_KERNEL_FLUX, false);
            return;
        }
        mark(ZSME_KERNEL_FLUX, true);
        const int gf = blocks_for(pm_.F, lc_.face);
        switch (lc_.face_occ) {
#define ZSME_FACE(OCC)                                                                                          \
    case OCC:                                                                                                   \
        face_kernel<M, N, OCC><<<gf, lc_.face, 0, stream_>>>(md_, 0, pm_.F, fs_cur_, aux_.p, params_.p, t_host,  \
                                                             t_dev, frac, dt, fb_.p, active);                   \
        break;
            ZSME_FACE(2) ZSME_FACE(3) ZSME_FACE(4)
            default: ZSME_FACE(1)
#undef ZSME_FACE
        }
        mark(ZSME_KERNEL_FLUX, false);
        if (face_only) return;
        mark(ZSME_KERNEL_GATHER, true);
        gather_kernel<M><<<blocks_for(pm_.C, lc_.gather), lc_.gather, 0, stream_>>>(md_, opts_, 0, pm_.C, fb_.p,
                                                                                   mode, x_in, x_out, base, dt,
                                                                                   active, aux_.p, params_.p, xl_out);
        mark(ZSME_KERNEL_GATHER, false);
    }
    // fg: the last SSP stage's gather, fused into the finalize kernel (or nullptr)
    void finalize_range(int c0, int cn, const StepDev& sd, const double* dt_src, int flags,
                        const FinalGather* fg = nullptr) {
        const int gb = blocks_for(cn, lc_.finalize);
        if (flags & FIN_SOURCE) cudaMemsetAsync(sd.n_fallback, 0, sizeof(int), stream_);
        mark(ZSME_KERNEL_FINALIZE, true);
        if (fg) {
            switch (lc_.finalize_occ) {
#define ZSME_FING(OCC)                                                                                           \
    case OCC:                                                                                                    \
        finalize_kernel<M, N, OCC, true><<<gb, lc_.finalize, 0, stream_>>>(md_, c0, cn, x_.p, aux_.p, params_.p,  \
                                                                           sd, dt_src, flags, *fg);              \
        break;
                ZSME_FING(2) ZSME_FING(3) ZSME_FING(4)
                default: ZSME_FING(1)
#undef ZSME_FING
            }
        } else {
            switch (lc_.finalize_occ) {
#define ZSME_FIN(OCC)                                                                                            \
    case OCC:                                                                                                    \
        finalize_kernel<M, N, OCC><<<gb, lc_.finalize, 0, stream_>>>(md_, c0, cn, x_.p, aux_.p, params_.p, sd,    \
                                                                     dt_src, flags);                             \
        break;
                ZSME_FIN(2) ZSME_FIN(3) ZSME_FIN(4)
                default: ZSME_FIN(1)
#undef ZSME_FIN
            }
        }
        mark(ZSME_KERNEL_FINALIZE, false);
        if (flags & FIN_SOURCE) {   // the cells whose Newton update needs the generic GEPP (usually none)
            mark(ZSME_KERNEL_FALLBACK, true);
            finalize_fallback_kernel<M, N><<<std::min(blocks_for(cn, 64), 8 * sm_count_), 64, 0, stream_>>>(
                md_, x_.p, aux_.p, params_.p, sd, dt_src, flags);
            mark(ZSME_KERNEL_FALLBACK, false);
        }
    }
    void launch_finalize(const StepDev& sd, const double* dt_src, int flags, const FinalGather* fg = nullptr) {
        finalize_range(0, pm_.C, sd, dt_src, flags, fg);
    }

    int rhs(double t, const double* x_aos, double* f_aos) override {
        if (n_inst_ != 1) return set_error(ZSME_ERR_ARG, "zsme_rhs needs a single-instance handle");
        const int C = pm_.C;
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, x_aos, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(tmp_b_.p, w_.p, old_of_new_.p, 0, C, C, NQ);
        clamp_kernel<M><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, 0, C, w_.p, aux_.p, params_.p, wl_.p);
        launch_prep(w_.p, wl_.p, nullptr);
        launch_flux(MODE_RHS, t, nullptr, 0.0, nullptr, tmp_a_.p, nullptr, nullptr, nullptr);
        ZSME_CUDA(cudaGetLastError());
        return get_soa(0, tmp_a_.p, NQ, f_aos, false);
    }

    int update_state() override {
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        launch_derivative_aux(x_.p, nullptr);
        launch_finalize(sd, nullptr, FIN_PRE | FIN_WRITE);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        x_clamped_ = true;
        return ZSME_OK;
    }

    int source(double dt) override {
        std::vector<double> d(n_inst_, dt);
        ZSME_CUDA(cudaMemcpyAsync(dt_aux_.p, d.data(), n_inst_ * sizeof(double), cudaMemcpyHostToDevice, stream_));
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        launch_finalize(sd, dt_aux_.p, FIN_SOURCE | FIN_WRITE);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        x_clamped_ = false;     // the Newton result is not clamped until the next step
        return ZSME_OK;
    }

    int compute_dt(int inst, double* dt) override {
        int rc = check_inst(inst);
        if (rc) return rc;
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        launch_finalize(sd, nullptr, FIN_DT);
        end_step_kernel<<<blocks_for(n_inst_, 128), 128, 0, stream_>>>(sd, 0, n_inst_, 2, 0.0, dt_aux_.p);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaMemcpyAsync(dt, dt_aux_.p + inst, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    // One time step of every instance (MUSCLSolver.hpp:140-188).
    // wl0: clamped copy of x_ for the first stage (x_ itself when x_ is constrained).
    // tape (adjoint replay): NQ x C slots receiving each stage state W_1 .. W_{s-1}
    // and the stage output X' before finalize (tape[0] = W_0 is the caller's copy),
    // then 2 NQ x F slots receiving each stage's face states
    void enqueue_step(const double* dts, const double* wl0, double* tape = nullptr) {
        const size_t tape_n = (size_t)NQ * pm_.C;
        const size_t fs_n = (size_t)2 * NQ * pm_.F;
        const int ns = st_.reconstruction_order < 2 ? 1 : st_.ssp_stages;
        // with a tape (adjoint replay) each stage's face states and stage state are
        // produced in their tape slots directly: slot k < s holds W_k, slot s the
        // stage result X', then one slot of face states per stage
        auto stage_fs = [&](int i) {
            fs_cur_ = tape ? tape + (size_t)(ns + 1) * tape_n + (size_t)i * fs_n : fs_.p;
            dec_cur_ = tape && st_.reconstruction_order >= 2
                           ? tape + (size_t)(ns + 1) * tape_n + (size_t)ns * fs_n + (size_t)i * dec_rows() * pm_.C
                           : nullptr;
        };
        StepDev sd = step_dev(dts);
        const double* t = sd.t;
        const double* dt = sd.dt_step;
        const int* act = sd.active;
        mark(ZSME_KERNEL_BEGIN, true);
        begin_step_kernel<<<blocks_for(n_inst_, 128), 128, 0, stream_>>>(sd, 0, n_inst_);
        mark(ZSME_KERNEL_BEGIN, false);
        const bool mood = st_.positivity == ZSME_POSITIVITY_MOOD;
        if (mood) cudaMemcpyAsync(xs_.p, x_.p, xs_.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
        // the last stage's gather inside finalize: separate face and gather
        // kernels at order 2, and the stage result not needed on its own
        // (MOOD inspects it, the adjoint's tape keeps it)
        const bool fuse_final = lc_.fuse_final && lc_.tile_faces == 0 && st_.reconstruction_order >= 2 && !mood &&
                                !tape && !deriv_.n && st_.time_integration == ZSME_TIME_SPLITTING;
        double* w_last = x_.p;   // the last stage's state
        const bool imex = st_.time_integration == ZSME_TIME_IMEX;
        if (imex) {
            enqueue_imex_stages(t, dt, act, wl0);
        } else if (st_.reconstruction_order < 2) {
            launch_derivative_aux(x_.p, act);       // FormRHS's UpdateState of the stage state
            stage_fs(0);
            launch_prep(x_.p, x_.p, act);
            launch_flux(MODE_EULER, 0.0, t, 0.0, nullptr, nullptr, x_.p, dt, act);
            if (tape)
                cudaMemcpyAsync(tape + tape_n, x_.p, tape_n * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
        } else {
            const int s = st_.ssp_stages;
            for (int i = 0; i < s - 1; ++i) {
                const double frac = i / (s - 1.);
                double* w_in = i == 0 ? x_.p : w_last;
                double* w_out = tape ? tape + (size_t)(i + 1) * tape_n : w_.p;
                launch_derivative_aux(w_in, act);   // FormRHS's UpdateState of the stage state
                stage_fs(i);
                // later stages get their clamped copy from gather
                launch_prep(w_in, i == 0 ? wl0 : wl_.p, act);
                launch_flux(i == 0 ? MODE_FIRST : MODE_MID, 0.0, t, frac, w_in, w_out, nullptr, dt, act, wl_.p);
                w_last = w_out;
            }
            launch_derivative_aux(w_last, act);
            stage_fs(s - 1);
            launch_prep(w_last, wl_.p, act);
            launch_flux(MODE_FINAL, 0.0, t, 1.0, w_last, nullptr, x_.p, dt, act, nullptr, fuse_final);
            if (tape)
                cudaMemcpyAsync(tape + (size_t)s * tape_n, x_.p, tape_n * sizeof(double), cudaMemcpyDeviceToDevice,
                                stream_);
        }
        fs_cur_ = fs_.p;
        dec_cur_ = nullptr;
        if (mood) {   // a-posteriori first-order override of troubled cells
            cudaMemsetAsync(iscal_.p + 6, 0, sizeof(int), stream_);
            mark(ZSME_KERNEL_MOOD, true);
            mood_detect_kernel<<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, 0, pm_.C, x_.p, sd, mood_list_.p,
                                                                           iscal_.p + 6);
            mark(ZSME_KERNEL_MOOD, false);
            mark(ZSME_KERNEL_MOOD, true);
            mood_kernel<M, N><<<std::min(blocks_for(pm_.C, 64), 8 * sm_count_), 64, 0, stream_>>>(
                md_, x_.p, xs_.p, aux_.p, params_.p, sd, mood_list_.p, iscal_.p + 6);
            mark(ZSME_KERNEL_MOOD, false);
        }
        // IMEX carries the source in its stages (MUSCLSolver.hpp:173-182)
        const int flags = FIN_PRE | FIN_POST | FIN_WRITE | FIN_DT | (st_.source && !imex ? FIN_SOURCE : 0);
        const FinalGather fg{fb_.p, w_last, sd.dt_step, st_.ssp_stages};
        // EnforcePhysicalConstraints' UpdateState: the derivative aux of the
        // transport result before the constraints and the source
        launch_derivative_aux(x_.p, act);
        launch_finalize(sd, sd.dt_step, flags, fuse_final ? &fg : nullptr);
        launch_derivative_aux(x_.p, act);           // PostStep's UpdateState
        mark(ZSME_KERNEL_END, true);
        end_step_kernel<<<blocks_for(n_inst_, 128), 128, 0, stream_>>>(sd, 0, n_inst_, 1, 0.0, nullptr);
        mark(ZSME_KERNEL_END, false);
    }
    // The IMEX strategy's transport + source update of one step (SolverStrategies.hpp:62-128,
    // additive Runge-Kutta 2E at the step's dt): G_j = FormRHS(Y_j) by the
    // prep / face / gather kernels in MODE_RHS, Y_0 = x_ with its implicit
    // source, two implicit stages solved per cell, then x_ updated in place.
    void enqueue_imex_stages(const double* t, const double* dt, const int* act, const double* wl0) {
        namespace K = ark2e;
        const int C = pm_.C, nb = blocks_for(C, 128);
        auto rhs = [&](double* y, const double* wl, double frac, double* g) {
            launch_derivative_aux(y, act);
            launch_prep(y, wl, act);
            launch_flux(MODE_RHS, 0.0, t, frac, nullptr, g, nullptr, dt, act);
        };
        rhs(x_.p, wl0, 0.0, imex_g_[0].p);
        imex_source_kernel<M><<<nb, 128, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, imex_s_[0].p, act);
        const ImexTerms t1{{imex_g_[0].p}, {imex_s_[0].p}, {K::a10}, {K::t10}, 1};
        imex_stage_kernel<M><<<blocks_for(C, 64), 64, 0, stream_>>>(md_, t1, x_.p, aux_.p, params_.p, dt, act,
                                                                    imex_y_[0].p, imex_s_[1].p, iscal_.p + 1);
        clamp_kernel<M><<<nb, 128, 0, stream_>>>(md_, 0, C, imex_y_[0].p, aux_.p, params_.p, wl_.p);
        rhs(imex_y_[0].p, wl_.p, K::c1, imex_g_[1].p);
        const ImexTerms t2{{imex_g_[0].p, imex_g_[1].p}, {imex_s_[0].p, imex_s_[1].p}, {K::a20, K::a21},
                           {K::t20, K::t21}, 2};
        imex_stage_kernel<M><<<blocks_for(C, 64), 64, 0, stream_>>>(md_, t2, x_.p, aux_.p, params_.p, dt, act,
                                                                    imex_y_[1].p, imex_s_[2].p, iscal_.p + 1);
        clamp_kernel<M><<<nb, 128, 0, stream_>>>(md_, 0, C, imex_y_[1].p, aux_.p, params_.p, wl_.p);
        rhs(imex_y_[1].p, wl_.p, K::c2, imex_g_[2].p);
        const ImexTerms tb{{imex_g_[0].p, imex_g_[1].p, imex_g_[2].p},
                           {imex_s_[0].p, imex_s_[1].p, imex_s_[2].p},
                           {K::b0, K::b1, K::b2},
                           {K::b0, K::b1, K::b2},
                           3};
        imex_final_kernel<M><<<nb, 128, 0, stream_>>>(md_, tb, x_.p, dt, act);
    }
    // ------------------------------------------------ fully implicit strategy
    // The Newton-Krylov iteration of one BDF step runs on the host around the
    // kernels of implicit_kernels.cuh; every reduction it reads is a
    // deterministic two-pass sum on the device.
    int imp_dot_blocks() const { return std::max(1, std::min(2 * sm_count_, blocks_for((long long)NQ * pm_.C, 256))); }
    long long imp_n() const { return (long long)NQ * pm_.C; }
    // V_k . w for k < nk into dev (device; imp_red_ by default) and out (host,
    // when given: a synchronisation)
    int imp_dots(const double* V, long long ld, int nk, const double* w, double* out, double* dev = nullptr) {
        const int nb = imp_dot_blocks();
        if (!dev) dev = imp_red_.p;
        imp_multi_dot_kernel<<<dim3(nb, nk), 256, 0, stream_>>>(imp_n(), nk, V, ld, w, imp_part_.p);
        imp_reduce_kernel<<<nk, 256, 0, stream_>>>(nk, nb, imp_part_.p, dev);
        ZSME_CUDA(cudaGetLastError());
        if (out) {
            ZSME_CUDA(cudaMemcpyAsync(out, dev, nk * sizeof(double), cudaMemcpyDeviceToHost, stream_));
            ZSME_CUDA(cudaStreamSynchronize(stream_));
        }
        return ZSME_OK;
    }
    int imp_norm(const double* w, double& out) {
        double d = 0.0;
        int rc = imp_dots(w, 0, 1, w, &d);
        out = std::sqrt(d);
        return rc;
    }
    void imp_lincomb(double a, const double* x, double b, const double* y, double* out) {
        imp_lincomb_kernel<<<blocks_for(imp_n(), 256), 256, 0, stream_>>>(imp_n(), a, x, b, y, out);
    }
    // F(t, y, Xdot) = (Xdot - S(y)) - R(y) (IFunctionWrapper) into f; t_dev:
    // the time in device memory (the step's), else t
    void imp_residual(double t, const double* y, const BdfTerms& b, double* f, const double* t_dev = nullptr) {
        const int C = pm_.C;
        clamp_kernel<M><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, 0, C, y, aux_.p, params_.p, wl_.p);
        launch_prep(y, wl_.p, nullptr);
        launch_flux(MODE_RHS, t, t_dev, 0.0, nullptr, imp_R_.p, nullptr, nullptr, nullptr);
        imp_residual_kernel<M><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, y, aux_.p, params_.p, imp_R_.p, b, f);
    }
    // the step's residual: time and BDF coefficients from imp_scal_
    BdfTerms imp_bdf() const {
        return BdfTerms{nullptr, imp_xn_.p, imp_xnm1_.p, 0.0, 0.0, 0.0, 1.0, imp_scal_.p + 2};
    }
    void imp_residual_step(const double* y, double* f) { imp_residual(0.0, y, imp_bdf(), f, imp_scal_.p); }
    void imp_drop_graphs() {
        for (auto& g : imp_graph_)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
    // P(t, y, a) (FormImplicitJacobian): the state clamped with its aux
    // (UpdateState), the face blocks, the diagonal blocks in assembly order
    void imp_assemble(double t, const double* y, double a) {
        const int C = pm_.C, F = pm_.F;
        imp_update_state_kernel<M><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, y, aux_.p, params_.p, imp_xl_.p,
                                                                          imp_al_.p);
        imp_face_jac_kernel<M, N><<<blocks_for(F, 128), 128, 0, stream_>>>(md_, imp_xl_.p, imp_al_.p, params_.p, t,
                                                                          imp_fj_.p);
        imp_cell_jac_kernel<M><<<blocks_for(C, 64), 64, 0, stream_>>>(md_, imp_xl_.p, imp_al_.p, params_.p, a,
                                                                      imp_fj_.p, imp_pd_.p);
    }
    // out = D^-1 (F(X + hv v) - F(X)) / hv, hv = sqrt(eps) sqrt(1 + |X|) / |v| (the
    // Walker-Pernice differencing parameter of PETSc's matrix-free Jacobian);
    // |X|, |v| and hv stay on the device
    void imp_apply(const double* v, double* out) {
        const long long n = imp_n();
        double* sc = imp_scal_.p;
        imp_dots(v, 0, 1, v, nullptr, sc + 6);
        imp_hv_kernel<<<1, 1, 0, stream_>>>(sc + 6, sc + 1, sc + 7);
        imp_perturb_kernel<<<blocks_for(n, 256), 256, 0, stream_>>>(n, x_.p, v, sc + 7, imp_xt_.p);
        imp_residual_step(imp_xt_.p, imp_Ft_.p);
        imp_diffquot_dev_kernel<<<blocks_for(n, 256), 256, 0, stream_>>>(n, imp_Ft_.p, imp_F_.p, sc + 7, out);
        imp_block_solve_kernel<NQ><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(pm_.C, imp_lu_.p, imp_piv_.p, out, out);
    }
    // Arnoldi step j: w = D^-1 J V_j, h = V_0..j . w (into imp_red_), w -= V h,
    // w.w (imp_scal_[8]), V_{j+1} = w / |w|.  Fixed pointers and device
    // scalars only, so it is captured once per handle as a CUDA graph.
    void imp_enqueue_arnoldi(int j) {
        const long long n = imp_n();
        double* w = imp_w_.p;
        imp_apply(imp_V_.p + (size_t)j * n, w);
        imp_dots(imp_V_.p, n, j + 1, w, nullptr);
        imp_multi_axpy_kernel<<<blocks_for(n, 256), 256, 0, stream_>>>(n, j + 1, imp_V_.p, n, imp_red_.p, w);
        imp_dots(w, 0, 1, w, nullptr, imp_scal_.p + 8);
        imp_normalize_kernel<<<blocks_for(n, 256), 256, 0, stream_>>>(n, imp_scal_.p + 8, w,
                                                                      imp_V_.p + (size_t)(j + 1) * n);
    }
    int imp_arnoldi(int j) {
        if (profiling_) {   // per-kernel timing records events: plain launches
            imp_enqueue_arnoldi(j);
            ZSME_CUDA(cudaGetLastError());
            return ZSME_OK;
        }
        if (!imp_graph_[j]) {
            cudaGraph_t g = nullptr;
            ZSME_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            imp_enqueue_arnoldi(j);
            ZSME_CUDA(cudaStreamEndCapture(stream_, &g));
            cudaError_t e = cudaGraphInstantiate(&imp_graph_[j], g, 0);
            cudaGraphDestroy(g);
            ZSME_CUDA(e);
        }
        ZSME_CUDA(cudaGraphLaunch(imp_graph_[j], stream_));
        return ZSME_OK;
    }
    // Left-preconditioned restarted GMRES (restart 30, classical Gram-Schmidt,
    // Givens rotations, zero initial guess) for (D^-1 J) d = D^-1 (-F) into
    // imp_d_; stops when the preconditioned residual is below 1e-5 of its
    // initial norm (PETSc's KSP defaults) or after 10000 iterations.
    int imp_gmres(int& its) {
        constexpr int m = kImpRestart;
        const long long n = imp_n();
        const int C = pm_.C;
        its = 0;
        ZSME_CUDA(cudaMemsetAsync(imp_d_.p, 0, n * sizeof(double), stream_));
        imp_lincomb(-1.0, imp_F_.p, 0.0, nullptr, imp_r0_.p);
        imp_block_solve_kernel<NQ><<<blocks_for(C, 128), 128, 0, stream_>>>(C, imp_lu_.p, imp_piv_.p, imp_r0_.p,
                                                                            imp_r0_.p);
        double beta = 0.0;
        int rc = imp_norm(imp_r0_.p, beta);
        if (rc) return rc;
        if (!(beta > 0.0)) return ZSME_OK;
        const double tol = std::max(1e-5 * beta, 1e-50);
        const double* r = imp_r0_.p;
        std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hcol(m + 1);
        while (true) {
            imp_lincomb(1.0 / beta, r, 0.0, nullptr, imp_V_.p);
            std::fill(g.begin(), g.end(), 0.0);
            g[0] = beta;
            int j = 0;
            bool done = false;
            for (; j < m;) {
                // one synchronisation per Arnoldi step: the projections and |w|^2 come back together
                if ((rc = imp_arnoldi(j))) return rc;
                double hn2 = 0.0;
                ZSME_CUDA(cudaMemcpyAsync(hcol.data(), imp_red_.p, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                                          stream_));
                ZSME_CUDA(cudaMemcpyAsync(&hn2, imp_scal_.p + 8, sizeof(double), cudaMemcpyDeviceToHost, stream_));
                ZSME_CUDA(cudaStreamSynchronize(stream_));
                const double hn = std::sqrt(hn2);
                for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
                H[(size_t)(j + 1) * m + j] = hn;
                for (int i = 0; i < j; ++i) {   // earlier rotations on the new column
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
                ++its;
                ++j;
                const double res = std::fabs(g[j]);
                if (res <= tol || !(hn > 0.0) || its >= 10000 || !std::isfinite(res)) {
                    done = true;
                    break;
                }
            }
            // y = H^-1 g over the j columns taken; d += V y
            for (int i = j - 1; i >= 0; --i) {
                double s = g[i];
                for (int k = i + 1; k < j; ++k) s -= H[(size_t)i * m + k] * y[k];
                y[i] = H[(size_t)i * m + i] != 0.0 ? s / H[(size_t)i * m + i] : 0.0;
            }
            ZSME_CUDA(cudaMemcpyAsync(imp_red_.p, y.data(), j * sizeof(double), cudaMemcpyHostToDevice, stream_));
            imp_multi_add_kernel<<<blocks_for(n, 256), 256, 0, stream_>>>(n, j, imp_V_.p, n, imp_red_.p, imp_d_.p);
            ZSME_CUDA(cudaGetLastError());
            if (done) break;
            // restart: r = D^-1 (-F) - D^-1 J d
            imp_apply(imp_d_.p, imp_w_.p);
            imp_lincomb(1.0, imp_r0_.p, -1.0, imp_w_.p, imp_r_.p);
            r = imp_r_.p;
            if ((rc = imp_norm(r, beta))) return rc;
            if (!(beta > tol)) break;
        }
        return ZSME_OK;
    }
    // One BDF step of size h from the state in x_ at time t0 (TSBDF order 2,
    // order 1 on the first step after a state is set; variable-step
    // coefficients with w = h / h_prev): Newton on F(t0 + h, X, Xdot(X)) = 0 from
    // X = X_n, stopping when |F| <= 1e-4 or |F| <= 1e-3 |F_0| (the SNES
    // tolerances MUSCLSolver.hpp:107-110 sets) or the update is below 1e-8 |X|,
    // at most 50 iterations; each iteration assembles the diagonal blocks at X,
    // solves by GMRES and backtracks (halving, at most 10 times) until
    // |F| <= (1 - 1e-4 lambda) |F_prev|; no such lambda ends Newton unconverged.
    int imp_step(double t0, double h) {
        const long long n = imp_n();
        const size_t bytes = n * sizeof(double);
        // history: X_{n-1} (the start of the previous step; X_n itself on the
        // first step, where its coefficient is zero) and X_n
        ZSME_CUDA(cudaMemcpyAsync(imp_xnm1_.p, imp_have_prev_ ? imp_xn_.p : x_.p, bytes, cudaMemcpyDeviceToDevice,
                                  stream_));
        ZSME_CUDA(cudaMemcpyAsync(imp_xn_.p, x_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
        double c0 = 1.0, c1 = -1.0, c2 = 0.0;
        if (imp_have_prev_) {
            const double w = h / imp_h_prev_;
            c0 = (1.0 + 2.0 * w) / (1.0 + w);
            c1 = -(1.0 + w);
            c2 = w * w / (1.0 + w);
        }
        const double shift = c0 / h;
        const double t1 = t0 + h;
        {
            const double sc[6] = {t1, 0.0, c0, c1, c2, h};
            ZSME_CUDA(cudaMemcpyAsync(imp_scal_.p, sc, sizeof(sc), cudaMemcpyHostToDevice, stream_));
            ZSME_CUDA(cudaStreamSynchronize(stream_));
        }
        imp_residual_step(x_.p, imp_F_.p);
        double fnorm = 0.0;
        int rc = imp_norm(imp_F_.p, fnorm);
        if (rc) return rc;
        const double fnorm0 = fnorm;
        int it = 0, gm_total = 0, halvings = 0, conv = 0;
        for (; it < 50; ++it) {
            if (fnorm <= 1e-4 || (it > 0 && fnorm <= 1e-3 * fnorm0)) { conv = 1; break; }
            if (!std::isfinite(fnorm)) break;
            if ((rc = imp_dots(x_.p, 0, 1, x_.p, nullptr, imp_scal_.p + 9))) return rc;
            imp_sqrt_kernel<<<1, 1, 0, stream_>>>(imp_scal_.p + 9, imp_scal_.p + 1);   // |X| for the differencing
            imp_assemble(t1, x_.p, shift);
            imp_block_lu_kernel<NQ><<<blocks_for(pm_.C, 64), 64, 0, stream_>>>(pm_.C, imp_pd_.p, imp_lu_.p,
                                                                              imp_piv_.p);
            int gm = 0;
            if ((rc = imp_gmres(gm))) return rc;
            gm_total += gm;
            double lambda = 1.0, ft = 0.0;
            bool descent = false;
            for (int ls = 0; ls < 10; ++ls) {
                imp_lincomb(1.0, x_.p, lambda, imp_d_.p, imp_xt_.p);
                imp_residual_step(imp_xt_.p, imp_Ft_.p);
                if ((rc = imp_norm(imp_Ft_.p, ft))) return rc;
                if (ft <= (1.0 - 1e-4 * lambda) * fnorm) { descent = true; break; }
                lambda *= 0.5;
                ++halvings;
            }
            if (!descent) break;   // the line search failed: Newton diverged
            ZSME_CUDA(cudaMemcpyAsync(x_.p, imp_xt_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
            ZSME_CUDA(cudaMemcpyAsync(imp_F_.p, imp_Ft_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
            fnorm = ft;
            double dnorm = 0.0, xn2 = 0.0;
            if ((rc = imp_norm(imp_d_.p, dnorm)) || (rc = imp_norm(x_.p, xn2))) return rc;
            if (lambda * dnorm <= 1e-8 * xn2) { conv = fnorm <= 1e-4 || fnorm <= 1e-3 * fnorm0 ? 1 : 2; ++it; break; }
        }
        imp_stats_[0] = it;
        imp_stats_[1] = gm_total;
        imp_stats_[2] = halvings;
        imp_stats_[3] = conv;
        if (!conv) {   // as PETSc's TSStep after a diverged SNES: nothing of the step is kept
            ZSME_CUDA(cudaMemcpyAsync(x_.p, imp_xn_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
            if (imp_have_prev_)   // the history as before the step
                ZSME_CUDA(cudaMemcpyAsync(imp_xn_.p, imp_xnm1_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
            ZSME_CUDA(cudaStreamSynchronize(stream_));
            return set_error(ZSME_ERR_SOLVE, "implicit step: Newton did not converge in 50 iterations");
        }
        imp_h_prev_ = h;
        imp_have_prev_ = true;
        return ZSME_OK;
    }
    // MUSCLSolver::Run with the implicit strategy: dt clamped to t_end, the BDF
    // step, the constraints (EnforcePhysicalConstraints), PostStep's
    // constraints and the next CFL dt.  Host-driven: no CUDA graph.
    int implicit_steps(int nsteps, const double* dts_host) {
        if (dts_host) {
            ZSME_CUDA(dts_.alloc((size_t)nsteps));
            ZSME_CUDA(cudaMemcpyAsync(dts_.p, dts_host, nsteps * sizeof(double), cudaMemcpyHostToDevice, stream_));
            ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, sizeof(int), stream_));
        }
        for (int i = 0; i < nsteps; ++i) {
            StepDev sd = step_dev(dts_host ? dts_.p : nullptr);
            begin_step_kernel<<<1, 32, 0, stream_>>>(sd, 0, 1);
            double t0 = 0.0, h = 0.0;
            int act = 0;
            ZSME_CUDA(cudaMemcpyAsync(&t0, t_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
            ZSME_CUDA(cudaMemcpyAsync(&h, dt_step_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
            ZSME_CUDA(cudaMemcpyAsync(&act, active_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
            ZSME_CUDA(cudaStreamSynchronize(stream_));
            if (!act) break;
            int rc = imp_step(t0, h);
            if (rc) return rc;
            launch_finalize(sd, nullptr, FIN_PRE | FIN_POST | FIN_DT | FIN_WRITE);
            end_step_kernel<<<1, 32, 0, stream_>>>(sd, 0, 1, 1, 0.0, nullptr);
            ZSME_CUDA(cudaGetLastError());
        }
        x_clamped_ = true;
        return collect_profile();
    }
    int implicit_stats(int* out) const override {
        for (int i = 0; i < 4; ++i) out[i] = imp_stats_[i];
        return ZSME_OK;
    }
    // F(t, X, Xdot) of caller states (AoS, caller order) into f_aos
    int implicit_function(double t, const double* x_aos, const double* xdot_aos, double* f_aos) override {
        if (st_.time_integration != ZSME_TIME_IMPLICIT)
            return set_error(ZSME_ERR_ARG, "the handle's time_integration is not ZSME_TIME_IMPLICIT");
        const int C = pm_.C;
        const size_t bytes = (size_t)NQ * C * sizeof(double);
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, x_aos, bytes, cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(tmp_b_.p, imp_xt_.p, old_of_new_.p, 0, C, C, NQ);
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, xdot_aos, bytes, cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(tmp_b_.p, imp_w_.p, old_of_new_.p, 0, C, C, NQ);
        const BdfTerms b{imp_w_.p, nullptr, nullptr, 0.0, 0.0, 0.0, 1.0, nullptr};
        imp_residual(t, imp_xt_.p, b, imp_Ft_.p);
        ZSME_CUDA(cudaGetLastError());
        return get_soa(0, imp_Ft_.p, NQ, f_aos, false);
    }
    // P(t, X, a) of a caller state: diagonal blocks [C][NQ][NQ] in caller
    // cell order, and per original face its blocks (row cell L, column R) and
    // (row R, column L), [F][2][NQ][NQ] (zero for boundary faces)
    int implicit_jacobian(double t, const double* x_aos, double a, double* diag, double* offdiag) override {
        if (st_.time_integration != ZSME_TIME_IMPLICIT)
            return set_error(ZSME_ERR_ARG, "the handle's time_integration is not ZSME_TIME_IMPLICIT");
        const int C = pm_.C, F = pm_.F;
        constexpr int Q2 = NQ * NQ;
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, x_aos, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(tmp_b_.p, imp_xt_.p, old_of_new_.p, 0, C, C, NQ);
        imp_assemble(t, imp_xt_.p, a);
        ZSME_CUDA(cudaGetLastError());
        std::vector<double> pd((size_t)Q2 * C), fj((size_t)4 * Q2 * F);
        ZSME_CUDA(cudaMemcpyAsync(pd.data(), imp_pd_.p, pd.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaMemcpyAsync(fj.data(), imp_fj_.p, fj.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        if (diag)
            for (int c = 0; c < C; ++c) {
                const int o = pm_.old_of_new[c];
                for (int e = 0; e < Q2; ++e) diag[(size_t)o * Q2 + e] = pd[(size_t)e * C + c];
            }
        if (offdiag)
            for (int f = 0; f < F; ++f) {
                const int o = pm_.face_old_of_new[f];
                const bool interior = pm_.face_R[f] >= 0 && pm_.farea[f] > 1e-15;
                for (int e = 0; e < Q2; ++e) {
                    // the matrix entry: zero plus the one block added there
                    offdiag[((size_t)o * 2 + 0) * Q2 + e] = interior ? 0.0 + fj[((size_t)f * 4 + 1) * Q2 + e] : 0.0;
                    offdiag[((size_t)o * 2 + 1) * Q2 + e] = interior ? 0.0 + fj[((size_t)f * 4 + 2) * Q2 + e] : 0.0;
                }
            }
        return ZSME_OK;
    }
    int launches_per_step() const override {
        if (st_.time_integration == ZSME_TIME_IMEX) {
            const int per_rhs = (lc_.tile_faces > 0 ? 2 : 3) + (deriv_.n ? 1 : 0);
            return 3 + 3 * per_rhs + 6 + (deriv_.n ? 2 : 0) + (st_.positivity == ZSME_POSITIVITY_MOOD ? 2 : 0);
        }
        const int per_stage = lc_.tile_faces > 0 ? 2 : 3;
        const bool fuse_final = lc_.fuse_final && lc_.tile_faces == 0 && st_.reconstruction_order >= 2 &&
                                st_.positivity != ZSME_POSITIVITY_MOOD && !deriv_.n;
        const int derivs = deriv_.n ? (st_.reconstruction_order < 2 ? 1 : st_.ssp_stages) + 2 : 0;
        return 3 + derivs - (fuse_final ? 1 : 0) +
               (st_.reconstruction_order < 2 ? per_stage : per_stage * st_.ssp_stages) +
               (st_.positivity == ZSME_POSITIVITY_MOOD ? 2 : 0) + (st_.source ? 1 : 0);
    }

    int step(int nsteps, const double* dts_host) override {
        if (nsteps <= 0) return ZSME_OK;
        if (dts_host && n_inst_ != 1) return set_error(ZSME_ERR_ARG, "imposed dts need a single-instance handle");
        if (st_.time_integration == ZSME_TIME_IMPLICIT) {
            ZSME_CUDA(cudaMemsetAsync(iscal_.p + 1, 0, 4 * sizeof(int), stream_));
            ZSME_CUDA(cudaMemsetAsync(iscal_.p + 7, 0, sizeof(int), stream_));
            return implicit_steps(nsteps, dts_host);
        }
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 1, 0, 4 * sizeof(int), stream_));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 7, 0, sizeof(int), stream_));
        // x_ is constrained after set_state, update_state and every step (update_variables is a
        // projection: the clamp of a clamped state is that state), so it serves as its own
        // clamped copy; after a bare source() the first step clamps a copy first, uncaptured
        const bool unclamped = !x_clamped_ && st_.reconstruction_order >= 2;
        x_clamped_ = true;
        if (unclamped)
            clamp_kernel<M><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, 0, pm_.C, x_.p, aux_.p, params_.p,
                                                                        wl_.p);
        if (dts_host || profiling_ || unclamped) {
            // imposed dts or per-kernel timing: plain launches (the step index
            // lives on the device)
            if (dts_host) {
                ZSME_CUDA(dts_.alloc((size_t)nsteps));
                ZSME_CUDA(cudaMemcpyAsync(dts_.p, dts_host, nsteps * sizeof(double), cudaMemcpyHostToDevice, stream_));
                ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, sizeof(int), stream_));
            }
            for (int i = 0; i < nsteps; ++i)
                enqueue_step(dts_host ? dts_.p : nullptr, (unclamped && i == 0) ? wl_.p : x_.p);
            ZSME_CUDA(cudaGetLastError());
            int rc = collect_profile();
            if (rc) return rc;
        } else {
            if (!graph_) {
                cudaGraph_t g = nullptr;
                ZSME_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
                enqueue_step(nullptr, x_.p);
                ZSME_CUDA(cudaStreamEndCapture(stream_, &g));
                ZSME_CUDA(cudaGraphInstantiate(&graph_, g, 0));
                cudaGraphDestroy(g);
            }
            for (int i = 0; i < nsteps; ++i) ZSME_CUDA(cudaGraphLaunch(graph_, stream_));
        }
        return ZSME_OK;
    }

    int step_device_dts(int nsteps, const double* d_dts) override {
        if (nsteps <= 0) return ZSME_OK;
        if (n_inst_ != 1) return set_error(ZSME_ERR_ARG, "imposed dts need a single-instance handle");
        if (st_.time_integration == ZSME_TIME_IMPLICIT)
            return set_error(ZSME_ERR_ARG, "device-resident dts need an explicit or IMEX time integration");
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 1, 0, 4 * sizeof(int), stream_));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 7, 0, sizeof(int), stream_));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, sizeof(int), stream_));   // index into d_dts
        const bool unclamped = !x_clamped_ && st_.reconstruction_order >= 2;
        x_clamped_ = true;
        if (unclamped)
            clamp_kernel<M><<<blocks_for(pm_.C, 128), 128, 0, stream_>>>(md_, 0, pm_.C, x_.p, aux_.p, params_.p,
                                                                        wl_.p);
        for (int i = 0; i < nsteps; ++i) enqueue_step(d_dts, (unclamped && i == 0) ? wl_.p : x_.p);
        ZSME_CUDA(cudaGetLastError());
        return collect_profile();
    }
    int get_time_device(double* d_t, double* d_dt) override {
        if (d_t) ZSME_CUDA(cudaMemcpyAsync(d_t, t_.p, sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        if (d_dt) ZSME_CUDA(cudaMemcpyAsync(d_dt, dt_cfl_.p, sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        return ZSME_OK;
    }

    // ------------------------------------------------------ discrete adjoint
    // R'(W)^T (factor * dt * src) + c_src * src -> dst for the stage state W with
    // face states fs.  dt = *dtp and the stage time *tp + frac * dt are device
    // scalars of the step, so that the launches of one checkpoint segment are the
    // same for every segment and replay as one CUDA graph.  W0: W is the step's
    // start state (its own clamped copy, as in the forward stage).
    void adj_apply_rt(const double* W, const double* fs, bool W0, const double* tp, double frac, const double* dtp,
                      double factor, const double* src, double c_src, double* dst,
                      const AdjEpilogue& ep = AdjEpilogue{}, const double* dec = nullptr) {
        const int C = pm_.C, F = pm_.F;
        const double* wl = W;
        if (!W0) {
            clamp_kernel<M><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, 0, C, W, adj_aux_cur_, params_.p, adj_wl_.p);
            wl = adj_wl_.p;
        }
        if constexpr (HasFluxVJP<N>::value) {   // the plugin's generated reverse sweep
            adj_face_vjp_kernel<MT, NT><<<blocks_for(F, 128), 128, 0, stream_>>>(md_, fs, adj_aux_cur_, params_.p, tp,
                                                                                frac, dtp, factor, src, adj_gfs_.p);
        } else {
            adj_face_kernel<MT, NT><<<blocks_for((long long)F * 2, 128), 128, 0, stream_>>>(
                md_, fs, adj_aux_cur_, params_.p, tp, frac, dtp, factor, src, adj_gfs_.p);
        }
        if (pm_.K == 3)
            adj_cell_kernel<MT, 3><<<blocks_for(C, 128), 128, 0, stream_>>>(
                md_, opts_, W, wl, params_.p, adj_gfs_.p, adj_own_w_.p, adj_own_wl_.p, adj_out_w_.p, adj_out_wl_.p,
                dec);
        else
            adj_cell_kernel<MT, 4><<<blocks_for(C, 128), 128, 0, stream_>>>(
                md_, opts_, W, wl, params_.p, adj_gfs_.p, adj_own_w_.p, adj_own_wl_.p, adj_out_w_.p, adj_out_wl_.p,
                dec);
        adj_combine_kernel<MT><<<blocks_for(C, 128), 128, 0, stream_>>>(md_, W, adj_aux_cur_, params_.p, adj_own_w_.p,
                                                                        adj_own_wl_.p, adj_out_w_.p, adj_out_wl_.p,
                                                                        src, c_src, dst, ep);
    }

    // Reverse of step k of the current segment (tape slot k: W_0 .. W_{s-1}, X',
    // then each stage's face states): adj_lam0_ holds the adjoint of X_{n+1}
    // and receives that of X_n, plus the seeds of the observations of X_n.
    void adj_step(int k) {
        const int C = pm_.C;
        const size_t nv = (size_t)NQ * C, fs_n = (size_t)2 * NQ * pm_.F;
        const size_t par = (size_t)adj_par_ * adj_tape_steps_;
        const double* tape = adj_tape_.p + (par + k) * adj_tstride_;
        const double* dtp = adj_seg_dt_.p + par + k;
        const double* tp = adj_seg_t_.p + par + k;
        double *lam = adj_lam0_.p, *t1 = adj_lam1_.p, *t2 = adj_lam2_.p;
        const int flags = FIN_PRE | FIN_POST | (st_.source ? FIN_SOURCE : 0);
        const int s = st_.reconstruction_order < 2 ? 1 : st_.ssp_stages;
        const int nb = blocks_for(C, 128);
        adj_finalize_kernel<MT><<<nb, 128, 0, stream_>>>(md_, tape + (size_t)s * nv, adj_aux_cur_, params_.p, dtp,
                                                         flags, lam, t1, adj_lp_cell_.p);
        // the observations of this step's start state, seeded by the last
        // combine where that one writes lam
        AdjEpilogue seeds;
        seeds.first = adj_first_.p;
        seeds.n0 = adj_seg_n0_.p + adj_par_;
        seeds.k = k;
        seeds.cell = adj_ocell_.p;
        seeds.comp = adj_ocomp_.p;
        seeds.seed = adj_oseed_.p;
        const double* fst = tape + (size_t)(s + 1) * nv;
        if (st_.reconstruction_order < 2) {  // X' = W0 + dt R(W0)
            adj_apply_rt(tape, fst, true, tp, 0.0, dtp, 1.0, t1, 1.0, lam, seeds);
            return;
        }
        // each stage's reconstruction record, after the face states
        const size_t dec_n = dec_rows() * C;
        const double* dect = fst + (size_t)s * fs_n;
        // X' = (s-1)/s W_{s-1} + dt/s R(W_{s-1}) + 1/s W_0
        adj_apply_rt(tape + (size_t)(s - 1) * nv, fst + (size_t)(s - 1) * fs_n, s - 1 == 0, tp, 1.0, dtp, 1.0 / s, t1,
                     (s - 1.) / s, t2, AdjEpilogue{}, dect + (size_t)(s - 1) * dec_n);
        double* cur = t2;
        double* oth = lam;
        for (int i = s - 2; i >= 0; --i) {  // W_{i+1} = W_i + dt/(s-1) R(W_i)
            AdjEpilogue ep;
            if (i == 0 && oth == lam) {     // the last combine writes lam: the W_0 share and the seeds with it
                ep = seeds;
                ep.ax_x = t1;
                ep.ax_a = 1.0 / s;
            }
            adj_apply_rt(tape + (size_t)i * nv, fst + (size_t)i * fs_n, i == 0, tp, i / (s - 1.), dtp,
                         1.0 / (s - 1.), cur, 1.0, oth, ep, dect + (size_t)i * dec_n);
            std::swap(cur, oth);
        }
        if (cur != lam) {   // odd s: the last combine wrote t2
            axpby_kernel<<<blocks_for((long long)nv, 256), 256, 0, stream_>>>((long long)nv, 1.0 / s, t1, 1.0, cur);
            cudaMemcpyAsync(lam, cur, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
            adj_seed_seg_kernel<<<1, 1, 0, stream_>>>(adj_first_.p, adj_seg_n0_.p + adj_par_, k, adj_ocell_.p,
                                                      adj_ocomp_.p, adj_oseed_.p, C, lam);
        }
    }

    // Replay of steps n0 .. n0+cnt-1 with the segment's dts into the tape
    // buffer adj_par_.
    void adj_replay(int cnt) {
        const size_t nv = (size_t)NQ * pm_.C;
        const size_t par = (size_t)adj_par_ * adj_tape_steps_;
        cudaMemsetAsync(iscal_.p, 0, sizeof(int), stream_);
        for (int k = 0; k < cnt; ++k) {
            double* tp = adj_tape_.p + (par + k) * adj_tstride_;
            cudaMemcpyAsync(tp, x_.p, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
            enqueue_step(adj_seg_dt_.p + par, x_.p, tp);
        }
    }
    void adj_reverse(int cnt) {
        for (int k = cnt - 1; k >= 0; --k) adj_step(k);
    }

    bool adjoint_overlapped() const override { return adj_overlapped_; }
    int adjoint_phases(double* ms) override {
        for (int i = 0; i < 3; ++i) ms[i] = adj_phase_ms_[i];
        return ZSME_OK;
    }

    int adjoint(const AdjointSpec& A, double* loss, double* grad_q, double* grad_p, double* dts_out) override {
        if (n_inst_ != 1) return set_error(ZSME_ERR_ARG, "the adjoint needs a single-instance handle");
        if (A.nsteps < 0 || A.every < 1 || A.nobs < 0)
            return set_error(ZSME_ERR_ARG, "adjoint: nsteps >= 0, checkpoint interval >= 1 and n_obs >= 0 required");
        if (A.nobs && (!A.obs_step || !A.obs_cell || !A.obs_comp || !A.obs_target))
            return set_error(ZSME_ERR_ARG, "adjoint: null observation array");
        if (!x_clamped_)
            return set_error(ZSME_ERR_STATE, "adjoint: the state is not constrained (call zsme_update_state)");
        if (st_.time_integration != ZSME_TIME_SPLITTING)
            return set_error(ZSME_ERR_ARG, "adjoint: only the splitting time integration is differentiated");
        if (st_.positivity != ZSME_POSITIVITY_NONE)
            return set_error(ZSME_ERR_ARG, "adjoint: the positivity variants are not differentiated (positivity none only)");
        const int C = pm_.C, F = pm_.F, K = pm_.K, NS = A.nsteps, E = A.every;
        const int s = st_.reconstruction_order < 2 ? 1 : st_.ssp_stages;
        const size_t nv = (size_t)NQ * C, na = (size_t)NA * C;
        // observations in device numbering, grouped by step (stable)
        std::vector<int> ord(A.nobs);
        for (int j = 0; j < A.nobs; ++j) {
            ord[j] = j;
            if (A.obs_step[j] < 0 || A.obs_step[j] > NS || A.obs_cell[j] < 0 || A.obs_cell[j] >= C ||
                A.obs_comp[j] < 0 || A.obs_comp[j] >= NQ)
                return set_error(ZSME_ERR_ARG, "adjoint: observation " + std::to_string(j) + " out of range");
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return A.obs_step[x] < A.obs_step[y]; });
        std::vector<int> first(NS + 2, 0), ocell(std::max(1, A.nobs), 0), ocomp(std::max(1, A.nobs), 0);
        for (int r = 0; r < A.nobs; ++r) {
            const int j = ord[r];
            ocell[r] = pm_.new_of_old[A.obs_cell[j]];
            ocomp[r] = A.obs_comp[j];
            first[A.obs_step[j] + 1]++;
        }
        for (int n = 0; n <= NS; ++n) first[n + 1] += first[n];
        const int nseg = (NS + E - 1) / E;
        std::vector<int> seg_n0(std::max(1, nseg));
        for (int g = 0; g < nseg; ++g) seg_n0[g] = g * E;
        ZSME_CUDA(adj_ocell_.upload(ocell, stream_));
        ZSME_CUDA(adj_ocomp_.upload(ocomp, stream_));
        ZSME_CUDA(adj_first_.upload(first, stream_));
        ZSME_CUDA(adj_segn0_all_.upload(seg_n0, stream_));
        ZSME_CUDA(adj_seg_n0_.alloc(2));
        ZSME_CUDA(adj_oval_.alloc(std::max(1, A.nobs)));
        ZSME_CUDA(adj_oseed_.alloc(std::max(1, A.nobs)));
        ZSME_CUDA(adj_ck_x_.alloc((size_t)(nseg + 1) * nv));
        ZSME_CUDA(adj_ck_a_.alloc((size_t)(nseg + 1) * na));
        // one step's tape: the stage states and the stage output, each stage's
        // face states, and at order 2 each stage's reconstruction record
        adj_tstride_ = (size_t)(s + 1) * nv + (size_t)s * 2 * NQ * F +
                       (st_.reconstruction_order >= 2 ? (size_t)s * dec_rows() * C : 0);
        const int tape_steps = std::min(E, std::max(NS, 1));
        // the replay of segment g-1 runs on a side stream while the reverse sweep
        // of segment g runs on the handle's stream: two tape buffers, CUDA graphs
        // for every segment (all segments full), and room for both buffers
        const size_t tape_bytes = (size_t)tape_steps * adj_tstride_ * sizeof(double);
        bool overlap = !profiling_ && nseg >= 2 && NS % E == 0;
        if (overlap) {
            size_t fr = 0, tot = 0;
            ZSME_CUDA(cudaMemGetInfo(&fr, &tot));
            const size_t held = adj_tape_.n * sizeof(double);
            overlap = fr + held >= 2 * tape_bytes + ((size_t)2 << 30);
        }
        if (overlap && !adj_side_) ZSME_CUDA(cudaStreamCreateWithFlags(&adj_side_, cudaStreamNonBlocking));
        adj_tape_steps_ = tape_steps;
        adj_overlapped_ = overlap;
        ZSME_CUDA(adj_tape_.alloc((size_t)(overlap ? 2 : 1) * tape_steps * adj_tstride_));
        ZSME_CUDA(adj_aux_snap_.alloc((size_t)2 * na));
        for (auto* b : {&adj_lam0_, &adj_lam1_, &adj_lam2_, &adj_own_w_, &adj_own_wl_, &adj_wl_})
            ZSME_CUDA(b->alloc(nv));
        ZSME_CUDA(adj_out_w_.alloc((size_t)K * nv));
        ZSME_CUDA(adj_out_wl_.alloc((size_t)K * nv));
        ZSME_CUDA(adj_gfs_.alloc((size_t)2 * NQ * F));
        ZSME_CUDA(adj_lp_cell_.alloc((size_t)NP * blocks_for(C, 128)));  // per-block partial sums
        ZSME_CUDA(adj_lp_.alloc(NP));
        ZSME_CUDA(adj_dts_.alloc(std::max(1, NS)));
        ZSME_CUDA(adj_th_.alloc((size_t)NS + 1));
        ZSME_CUDA(adj_seg_dt_.alloc((size_t)2 * tape_steps));
        ZSME_CUDA(adj_seg_t_.alloc((size_t)2 * tape_steps));
        auto obs_values = [&](int n) {
            const int cnt = first[n + 1] - first[n];
            if (cnt > 0)
                obs_value_kernel<<<blocks_for(cnt, 128), 128, 0, stream_>>>(cnt, adj_ocell_.p + first[n],
                                                                            adj_ocomp_.p + first[n], x_.p, C,
                                                                            adj_oval_.p + first[n]);
        };
        auto save = [&](int slot) {
            cudaMemcpyAsync(adj_ck_x_.p + (size_t)slot * nv, x_.p, nv * sizeof(double), cudaMemcpyDeviceToDevice, stream_);
            cudaMemcpyAsync(adj_ck_a_.p + (size_t)slot * na, aux_.p, na * sizeof(double), cudaMemcpyDeviceToDevice,
                            stream_);
        };
        auto restore = [&](int slot, cudaStream_t st) {
            cudaMemcpyAsync(x_.p, adj_ck_x_.p + (size_t)slot * nv, nv * sizeof(double), cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(aux_.p, adj_ck_a_.p + (size_t)slot * na, na * sizeof(double), cudaMemcpyDeviceToDevice, st);
        };
        cudaEvent_t ev[4];
        for (auto& e : ev) ZSME_CUDA(cudaEventCreate(&e));
        struct EvGuard {
            cudaEvent_t* e;
            ~EvGuard() { for (int i = 0; i < 4; ++i) cudaEventDestroy(e[i]); }
        } ev_guard{ev};
        // ---- forward: CFL steps, checkpoints, observed values, dt record
        double t0 = 0.0;
        ZSME_CUDA(cudaMemcpyAsync(&t0, t_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        ZSME_CUDA(cudaEventRecord(ev[0], stream_));
        save(0);
        for (int n = 0; n < NS; ++n) {
            obs_values(n);
            int rc = step(1, nullptr);
            if (rc) return rc;
            ZSME_CUDA(cudaMemcpyAsync(adj_dts_.p + n, dt_step_.p, sizeof(double), cudaMemcpyDeviceToDevice, stream_));
            if ((n + 1) % E == 0 && n + 1 < NS) save((n + 1) / E);
        }
        obs_values(NS);
        save(nseg);  // the final state, restored at the end
        ZSME_CUDA(cudaEventRecord(ev[1], stream_));
        double t_fin = 0.0, dtc_fin = 0.0;
        std::vector<double> dth(std::max(1, NS)), oval(std::max(1, A.nobs));
        ZSME_CUDA(cudaMemcpyAsync(&t_fin, t_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaMemcpyAsync(&dtc_fin, dt_cfl_.p, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaMemcpyAsync(dth.data(), adj_dts_.p, dth.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaMemcpyAsync(oval.data(), adj_oval_.p, oval.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                  stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        {
            float a0 = 0.f;
            ZSME_CUDA(cudaEventElapsedTime(&a0, ev[0], ev[1]));
            adj_phase_ms_[0] = a0;
        }
        // step start times as the device forms them (t += dt)
        std::vector<double> th(NS + 1);
        th[0] = t0;
        for (int n = 0; n < NS; ++n) th[n + 1] = th[n] + dth[n];
        ZSME_CUDA(cudaMemcpyAsync(adj_th_.p, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
        // loss in the caller's order; seeds 2 w (q - target) in device order
        std::vector<double> val_of(A.nobs), seed(std::max(1, A.nobs), 0.0);
        for (int r = 0; r < A.nobs; ++r) val_of[ord[r]] = oval[r];
        double L = 0.0;
        for (int j = 0; j < A.nobs; ++j) {
            const double wj = A.obs_weight ? A.obs_weight[j] : 1.0;
            const double rr = val_of[j] - A.obs_target[j];
            L += wj * rr * rr;
        }
        for (int r = 0; r < A.nobs; ++r) {
            const int j = ord[r];
            seed[r] = 2.0 * (A.obs_weight ? A.obs_weight[j] : 1.0) * (val_of[j] - A.obs_target[j]);
        }
        ZSME_CUDA(cudaMemcpyAsync(adj_oseed_.p, seed.data(), seed.size() * sizeof(double), cudaMemcpyHostToDevice,
                                  stream_));
        // ---- reverse, segment by segment; full segments replay captured graphs
        ZSME_CUDA(cudaMemsetAsync(adj_lam0_.p, 0, nv * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(adj_lp_.p, 0, NP * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(adj_lp_cell_.p, 0, adj_lp_cell_.n * sizeof(double), stream_));
        {
            const int cnt = first[NS + 1] - first[NS];
            if (cnt > 0)
                adj_seed_kernel<<<1, 1, 0, stream_>>>(cnt, adj_ocell_.p + first[NS], adj_ocomp_.p + first[NS],
                                                      adj_oseed_.p + first[NS], C, adj_lam0_.p);
        }
        const bool graphs = !profiling_;
        cudaGraphExec_t gx[4] = {nullptr, nullptr, nullptr, nullptr};   // replay, reverse per tape buffer
        struct GraphGuard {
            cudaGraphExec_t* g;
            ~GraphGuard() {
                for (int i = 0; i < 4; ++i)
                    if (g[i]) cudaGraphExecDestroy(g[i]);
            }
        } graph_guard{gx};
        auto capture = [&](cudaGraphExec_t* out, bool replay) -> int {
            cudaGraph_t gr = nullptr;
            ZSME_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            if (replay) adj_replay(E);
            else adj_reverse(E);
            ZSME_CUDA(cudaStreamEndCapture(stream_, &gr));
            cudaError_t e = cudaGraphInstantiate(out, gr, 0);
            cudaGraphDestroy(gr);
            ZSME_CUDA(e);
            return ZSME_OK;
        };
        // the segment's start time, dts, step times and first step index into buffer par
        auto seg_scalars = [&](int seg, int par, int cnt, cudaStream_t st) -> int {
            const int n0 = seg * E;
            const size_t o = (size_t)par * tape_steps;
            ZSME_CUDA(cudaMemcpyAsync(t_.p, adj_th_.p + n0, sizeof(double), cudaMemcpyDeviceToDevice, st));
            ZSME_CUDA(cudaMemcpyAsync(adj_seg_dt_.p + o, adj_dts_.p + n0, cnt * sizeof(double),
                                      cudaMemcpyDeviceToDevice, st));
            ZSME_CUDA(cudaMemcpyAsync(adj_seg_t_.p + o, adj_th_.p + n0, cnt * sizeof(double),
                                      cudaMemcpyDeviceToDevice, st));
            ZSME_CUDA(cudaMemcpyAsync(adj_seg_n0_.p + par, adj_segn0_all_.p + seg, sizeof(int),
                                      cudaMemcpyDeviceToDevice, st));
            return ZSME_OK;
        };
        float replay_ms = 0.f, reverse_ms = 0.f;
        if (!overlap) {
            // one tape buffer: replay, then reverse, segment by segment; the
            // reverse reads the aux array as the replay left it
            adj_par_ = 0;
            adj_aux_cur_ = aux_.p;
            for (int seg = nseg - 1; seg >= 0; --seg) {
                const int n0 = seg * E, cnt = std::min(NS, n0 + E) - n0;
                const bool full = cnt == E && graphs;
                ZSME_CUDA(cudaEventRecord(ev[2], stream_));
                restore(seg, stream_);
                int rc = seg_scalars(seg, 0, cnt, stream_);
                if (rc) return rc;
                if (full) {
                    if (!gx[0] && (rc = capture(&gx[0], true))) return rc;
                    ZSME_CUDA(cudaGraphLaunch(gx[0], stream_));
                } else {
                    adj_replay(cnt);
                }
                ZSME_CUDA(cudaEventRecord(ev[3], stream_));
                if (full) {
                    if (!gx[2] && (rc = capture(&gx[2], false))) return rc;
                    ZSME_CUDA(cudaGraphLaunch(gx[2], stream_));
                } else {
                    adj_reverse(cnt);
                }
                ZSME_CUDA(cudaGetLastError());
                ZSME_CUDA(cudaEventRecord(ev[1], stream_));
                ZSME_CUDA(cudaEventSynchronize(ev[1]));
                float a1 = 0.f, a2 = 0.f;
                ZSME_CUDA(cudaEventElapsedTime(&a1, ev[2], ev[3]));
                ZSME_CUDA(cudaEventElapsedTime(&a2, ev[3], ev[1]));
                replay_ms += a1;
                reverse_ms += a2;
            }
        } else {
            // two tape buffers: segment g's replay (side stream) fills buffer g % 2
            // while the handle's stream runs the reverse sweep of segment g + 1 out
            // of the other one.  Every segment is full, so the four graphs are
            // captured once, up front.  The reverse reads the aux snapshot taken
            // at the end of its own segment's replay, the array the one-buffer
            // form reads at that point.
            int rc = 0;
            for (int par = 0; par < 2; ++par) {
                adj_par_ = par;
                adj_aux_cur_ = adj_aux_snap_.p + (size_t)par * na;
                if ((rc = capture(&gx[par], true)) || (rc = capture(&gx[2 + par], false))) return rc;
            }
            cudaEvent_t ov[5];   // replay done (2), reverse done (2), start
            int made = 0;
            struct OvGuard {
                cudaEvent_t* e;
                int* n;
                ~OvGuard() { for (int i = 0; i < *n; ++i) cudaEventDestroy(e[i]); }
            } ov_guard{ov, &made};
            for (; made < 5; ++made) ZSME_CUDA(cudaEventCreateWithFlags(&ov[made], cudaEventDisableTiming));
            ZSME_CUDA(cudaEventRecord(ev[2], stream_));
            ZSME_CUDA(cudaEventRecord(ov[4], stream_));
            ZSME_CUDA(cudaStreamWaitEvent(adj_side_, ov[4], 0));
            bool rev_issued[2] = {false, false};
            for (int seg = nseg - 1; seg >= 0; --seg) {
                const int par = seg & 1;
                if (rev_issued[par]) ZSME_CUDA(cudaStreamWaitEvent(adj_side_, ov[2 + par], 0));
                restore(seg, adj_side_);
                if ((rc = seg_scalars(seg, par, E, adj_side_))) return rc;
                ZSME_CUDA(cudaGraphLaunch(gx[par], adj_side_));
                ZSME_CUDA(cudaMemcpyAsync(adj_aux_snap_.p + (size_t)par * na, aux_.p, na * sizeof(double),
                                          cudaMemcpyDeviceToDevice, adj_side_));
                ZSME_CUDA(cudaEventRecord(ov[par], adj_side_));
                ZSME_CUDA(cudaStreamWaitEvent(stream_, ov[par], 0));
                if (seg == nseg - 1) ZSME_CUDA(cudaEventRecord(ev[3], stream_));   // the first replay is exposed
                ZSME_CUDA(cudaGraphLaunch(gx[2 + par], stream_));
                ZSME_CUDA(cudaEventRecord(ov[2 + par], stream_));
                rev_issued[par] = true;
            }
            ZSME_CUDA(cudaGetLastError());
            ZSME_CUDA(cudaEventRecord(ev[1], stream_));
            ZSME_CUDA(cudaEventSynchronize(ev[1]));
            ZSME_CUDA(cudaEventElapsedTime(&replay_ms, ev[2], ev[3]));
            ZSME_CUDA(cudaEventElapsedTime(&reverse_ms, ev[3], ev[1]));
        }
        adj_phase_ms_[1] = replay_ms;
        adj_phase_ms_[2] = reverse_ms;
        // the parameter adjoint: the per-block sums over all steps, over the blocks
        adj_param_reduce_kernel<<<NP, 256, 0, stream_>>>(adj_lp_cell_.p, blocks_for(C, 128), adj_lp_.p);
        ZSME_CUDA(cudaGetLastError());
        // ---- outputs; the handle keeps the final state of the forward run
        if (grad_q) {
            int rc = get_soa(0, adj_lam0_.p, NQ, grad_q, false);
            if (rc) return rc;
        }
        if (grad_p) ZSME_CUDA(cudaMemcpyAsync(grad_p, adj_lp_.p, NP * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        restore(nseg, stream_);
        ZSME_CUDA(cudaMemcpyAsync(t_.p, &t_fin, sizeof(double), cudaMemcpyHostToDevice, stream_));
        ZSME_CUDA(cudaMemcpyAsync(dt_cfl_.p, &dtc_fin, sizeof(double), cudaMemcpyHostToDevice, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        if (loss) *loss = L;
        if (dts_out)
            for (int n = 0; n < NS; ++n) dts_out[n] = dth[n];
        x_clamped_ = true;
        return ZSME_OK;
    }

    int sync(int inst, zsme_diag* d) override {
        int rc = check_inst(inst);
        if (rc) return rc;
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        if (h2d_) {
            ZSME_CUDA(cudaStreamSynchronize(h2d_));
            ZSME_CUDA(cudaStreamSynchronize(d2h_));
        }
        double tt = 0, dd = 0;
        int is[8];
        ZSME_CUDA(cudaMemcpy(&tt, t_.p + inst, sizeof(double), cudaMemcpyDeviceToHost));
        ZSME_CUDA(cudaMemcpy(&dd, dt_cfl_.p + inst, sizeof(double), cudaMemcpyDeviceToHost));
        ZSME_CUDA(cudaMemcpy(is, iscal_.p, 8 * sizeof(int), cudaMemcpyDeviceToHost));
        if (d) {
            d->steps = is[0];
            d->time = tt;
            d->dt = dd;
            d->n_nonfinite = is[1];
            d->n_negative_depth = is[2];
            d->n_newton_unconverged = is[3];
            d->n_mood_cells = is[4];
            d->n_newton_deferred = is[7];
        }
        return ZSME_OK;
    }

    void* stream() override { return (void*)stream_; }
};

}  // namespace zsme

#define ZSME_DEFINE_MODEL(NS)                                                                 \
    zsme::SolverBase* zsme_make_##NS() { return new zsme::Solver<NS::Model, NS::Numerics>(); } \
    void zsme_info_##NS(int* v) {                                                             \
        v[0] = NS::Model<double>::n_dof_q;                                                    \
        v[1] = NS::Model<double>::n_dof_qaux;                                                 \
        v[2] = NS::Model<double>::n_parameters;                                               \
        v[3] = NS::Model<double>::dimension;                                                  \
    }
