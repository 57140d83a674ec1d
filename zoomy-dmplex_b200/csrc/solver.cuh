// Host side of one model's solver: device buffers, the CUDA stream, the
// captured CUDA graph of one time step, and the calls behind the C ABI.
// A solver advances one or several independent instances (an ensemble of
// meshes, concatenated cell- and face-wise); every kernel launch covers all
// instances.  Included once per model translation unit after the plugin.
#pragma once
#include <cuda_runtime.h>

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
    DevBuf<int> cell_inst_, face_inst_;
    DevBuf<double> slot_dx_, slot_w_, vol_, rc_, fn_, farea_, fc_, fnr_;
    // state
    DevBuf<double> x_, w_, aux_, fs_, fb_, tmp_a_, tmp_b_, params_, dts_;
    // per instance: t, dt_cfl, dt_step, dt_aux ; active ; ratio
    DevBuf<double> t_, dt_cfl_, dt_step_, dt_aux_;
    DevBuf<int> active_, iscal_;  // iscal_: [0] step_idx, [1..3] diag
    DevBuf<unsigned long long> ratio_;
    MeshDev md_{};
    Opts opts_{};
    // per-kernel CUDA-event timing (zsme_set_profiling)
    bool profiling_ = false;
    std::vector<cudaEvent_t> ev_pool_;
    std::vector<int> ev_kind_;
    size_t ev_used_ = 0;
    double prof_ms_[ZSME_KERNEL_KINDS] = {0};
    int64_t prof_n_[ZSME_KERNEL_KINDS] = {0};

  public:
    ~Solver() override {
        if (graph_) cudaGraphExecDestroy(graph_);
        for (auto e : ev_pool_) cudaEventDestroy(e);
        if (stream_) cudaStreamDestroy(stream_);
    }

    int n_dof_q() const override { return NQ; }
    int n_dof_qaux() const override { return NA; }
    int n_instances() const override { return n_inst_; }

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
        for (int o : {lc.prep_occ, lc.face_occ})
            if (o < 1 || o > 4) return set_error(ZSME_ERR_ARG, "occupancy caps must be 1..4 blocks per SM");
        lc_ = lc;
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
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
        ZSME_CUDA(cudaSetDevice(device_));
        ZSME_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        LaunchConfig lc{128, 128, 128, 128};
        if (st_.block_size > 0) lc.prep = lc.face = lc.gather = st_.block_size;
        int rc = set_launch(lc);
        if (rc) return rc;
        const int C = pm_.C, F = pm_.F;
        ZSME_CUDA(slot_nbr_.upload(pm_.slot_nbr, stream_));
        ZSME_CUDA(slot_meta_.upload(pm_.slot_meta, stream_));
        ZSME_CUDA(slot_face_.upload(pm_.slot_face, stream_));
        ZSME_CUDA(order_.upload(pm_.order, stream_));
        ZSME_CUDA(old_of_new_.upload(pm_.old_of_new, stream_));
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
        ZSME_CUDA(aux_.alloc((size_t)NA * C));
        ZSME_CUDA(fs_.alloc((size_t)2 * NQ * F));
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
        return ZSME_OK;
    }

    StepDev step_dev(const double* dts) {
        return StepDev{t_.p, dt_cfl_.p, dt_step_.p, active_.p, ratio_.p, dts, iscal_.p + 0, n_inst_,
                       st_.t_end, st_.cfl, M::dt_max, iscal_.p + 1};
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
        for (int k = 0; k < NA; ++k)
            ZSME_CUDA(cudaMemsetAsync(aux_.p + (size_t)k * pm_.C + c0, 0, cn * sizeof(double), stream_));
        ZSME_CUDA(cudaMemcpyAsync(t_.p + inst, &t, sizeof(double), cudaMemcpyHostToDevice, stream_));
        ZSME_CUDA(cudaMemsetAsync(active_.p + inst, 0, sizeof(int), stream_));
        if (inst == 0) ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, 8 * sizeof(int), stream_));
        // constraints, then dt_start = max(ComputeTimeStep, min_dt)
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        finalize_kernel<M, N><<<blocks_for(cn, lc_.finalize), lc_.finalize, 0, stream_>>>(
            md_, c0, cn, x_.p, aux_.p, params_.p, sd, nullptr, FIN_POST | FIN_WRITE | FIN_DT);
        ZSME_CUDA(cudaGetLastError());
        end_step_kernel<<<1, 32, 0, stream_>>>(step_dev(nullptr), inst, 1, 0, st_.min_dt, nullptr);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
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
    void launch_prep(const double* w, const int* active) {
        mark(ZSME_KERNEL_PREP, true);
        const int gb = blocks_for(pm_.C, lc_.prep);
        switch (lc_.prep_occ) {
#define ZSME_PREP(OCC)                                                                                          \
    case OCC:                                                                                                   \
        prep_kernel<M, OCC><<<gb, lc_.prep, 0, stream_>>>(md_, opts_, 0, pm_.C, w, aux_.p, params_.p, fs_.p,     \
                                                          active);                                              \
        break;
            ZSME_PREP(2) ZSME_PREP(3) ZSME_PREP(4)
            default: ZSME_PREP(1)
#undef ZSME_PREP
        }
        mark(ZSME_KERNEL_PREP, false);
    }
    void launch_flux(int mode, double t_host, const double* t_dev, double frac, const double* x_in, double* x_out,
                     double* base, const double* dt, const int* active) {
        mark(ZSME_KERNEL_FLUX, true);
        const int gf = blocks_for(pm_.F, lc_.face);
        switch (lc_.face_occ) {
#define ZSME_FACE(OCC)                                                                                          \
    case OCC:                                                                                                   \
        face_kernel<M, N, OCC><<<gf, lc_.face, 0, stream_>>>(md_, 0, pm_.F, fs_.p, aux_.p, params_.p, t_host,    \
                                                             t_dev, frac, dt, fb_.p, active);                   \
        break;
            ZSME_FACE(2) ZSME_FACE(3) ZSME_FACE(4)
            default: ZSME_FACE(1)
#undef ZSME_FACE
        }
        mark(ZSME_KERNEL_FLUX, false);
        mark(ZSME_KERNEL_GATHER, true);
        gather_kernel<M><<<blocks_for(pm_.C, lc_.gather), lc_.gather, 0, stream_>>>(md_, opts_, 0, pm_.C, fb_.p,
                                                                                   mode, x_in, x_out, base, dt,
                                                                                   active);
        mark(ZSME_KERNEL_GATHER, false);
    }
    void launch_finalize(const StepDev& sd, const double* dt_src, int flags) {
        mark(ZSME_KERNEL_FINALIZE, true);
        finalize_kernel<M, N><<<blocks_for(pm_.C, lc_.finalize), lc_.finalize, 0, stream_>>>(
            md_, 0, pm_.C, x_.p, aux_.p, params_.p, sd, dt_src, flags);
        mark(ZSME_KERNEL_FINALIZE, false);
    }

    int rhs(double t, const double* x_aos, double* f_aos) override {
        if (n_inst_ != 1) return set_error(ZSME_ERR_ARG, "zsme_rhs needs a single-instance handle");
        const int C = pm_.C;
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, x_aos, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<blocks_for(C, 128), 128, 0, stream_>>>(tmp_b_.p, w_.p, old_of_new_.p, 0, C, C, NQ);
        launch_prep(w_.p, nullptr);
        launch_flux(MODE_RHS, t, nullptr, 0.0, nullptr, tmp_a_.p, nullptr, nullptr, nullptr);
        ZSME_CUDA(cudaGetLastError());
        return get_soa(0, tmp_a_.p, NQ, f_aos, false);
    }

    int update_state() override {
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        launch_finalize(sd, nullptr, FIN_PRE | FIN_WRITE);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
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
    void enqueue_step(const double* dts) {
        StepDev sd = step_dev(dts);
        const double* t = sd.t;
        const double* dt = sd.dt_step;
        const int* act = sd.active;
        mark(ZSME_KERNEL_BEGIN, true);
        begin_step_kernel<<<blocks_for(n_inst_, 128), 128, 0, stream_>>>(sd, 0, n_inst_);
        mark(ZSME_KERNEL_BEGIN, false);
        if (st_.reconstruction_order < 2) {
            launch_prep(x_.p, act);
            launch_flux(MODE_EULER, 0.0, t, 0.0, nullptr, nullptr, x_.p, dt, act);
        } else {
            const int s = st_.ssp_stages;
            for (int i = 0; i < s - 1; ++i) {
                const double frac = i / (s - 1.);
                launch_prep(i == 0 ? x_.p : w_.p, act);
                launch_flux(i == 0 ? MODE_FIRST : MODE_MID, 0.0, t, frac, i == 0 ? x_.p : w_.p, w_.p, nullptr, dt,
                            act);
            }
            launch_prep(w_.p, act);
            launch_flux(MODE_FINAL, 0.0, t, 1.0, w_.p, nullptr, x_.p, dt, act);
        }
        const int flags = FIN_PRE | FIN_POST | FIN_WRITE | FIN_DT | (st_.source ? FIN_SOURCE : 0);
        launch_finalize(sd, sd.dt_step, flags);
        mark(ZSME_KERNEL_END, true);
        end_step_kernel<<<blocks_for(n_inst_, 128), 128, 0, stream_>>>(sd, 0, n_inst_, 1, 0.0, nullptr);
        mark(ZSME_KERNEL_END, false);
    }
    int launches_per_step() const override {
        return 3 + (st_.reconstruction_order < 2 ? 3 : 3 * st_.ssp_stages);
    }

    int step(int nsteps, const double* dts_host) override {
        if (nsteps <= 0) return ZSME_OK;
        if (dts_host && n_inst_ != 1) return set_error(ZSME_ERR_ARG, "imposed dts need a single-instance handle");
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 1, 0, 3 * sizeof(int), stream_));
        if (dts_host || profiling_) {
            // imposed dts or per-kernel timing: plain launches (the step index
            // lives on the device)
            if (dts_host) {
                ZSME_CUDA(dts_.alloc((size_t)nsteps));
                ZSME_CUDA(cudaMemcpyAsync(dts_.p, dts_host, nsteps * sizeof(double), cudaMemcpyHostToDevice, stream_));
                ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, sizeof(int), stream_));
            }
            for (int i = 0; i < nsteps; ++i) enqueue_step(dts_host ? dts_.p : nullptr);
            ZSME_CUDA(cudaGetLastError());
            int rc = collect_profile();
            if (rc) return rc;
        } else {
            if (!graph_) {
                cudaGraph_t g = nullptr;
                ZSME_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
                enqueue_step(nullptr);
                ZSME_CUDA(cudaStreamEndCapture(stream_, &g));
                ZSME_CUDA(cudaGraphInstantiate(&graph_, g, 0));
                cudaGraphDestroy(g);
            }
            for (int i = 0; i < nsteps; ++i) ZSME_CUDA(cudaGraphLaunch(graph_, stream_));
        }
        return ZSME_OK;
    }

    int sync(int inst, zsme_diag* d) override {
        int rc = check_inst(inst);
        if (rc) return rc;
        ZSME_CUDA(cudaStreamSynchronize(stream_));
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
            d->reserved = 0;
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
