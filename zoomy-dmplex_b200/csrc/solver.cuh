// Host side of one model's solver: device buffers, the CUDA stream, the
// captured CUDA graph of one time step, and the calls behind the C ABI.
// Included once per model translation unit after the model plugin.
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

template <template <typename> class MT, template <typename> class NT>
class Solver final : public SolverBase {
    using M = MT<double>;
    using N = NT<double>;
    static constexpr int NQ = M::n_dof_q, NA = M::n_dof_qaux, NP = M::n_parameters, DIM = M::dimension;

    PreparedMesh pm_;
    zsme_settings st_{};
    int device_ = 0, block_ = 128, grid_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    // mesh
    DevBuf<int> slot_nbr_, slot_meta_, slot_face_, order_, old_of_new_;
    DevBuf<double> slot_dx_, slot_w_, vol_, rc_, fn_, farea_, fc_, fnr_;
    // state
    DevBuf<double> x_, w_, aux_, fs_, tmp_a_, tmp_b_, params_, scal_, partial_, dts_;
    DevBuf<int> iscal_;
    MeshDev md_{};
    Opts opts_{};
    int64_t steps_ = 0;
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

    // Event pair around one launch when profiling (outside graph capture).
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

    int n_dof_q() const override { return NQ; }
    int n_dof_qaux() const override { return NA; }

    int init(PreparedMesh&& pm, const zsme_settings& st, const double* params, int device) override {
        pm_ = std::move(pm);
        st_ = st;
        device_ = device;
        if (pm_.dim != DIM) return set_error(ZSME_ERR_ARG, "mesh dimension does not match the model");
        if (st_.reconstruction_order >= 2 && st_.ssp_stages < 2)
            return set_error(ZSME_ERR_ARG, "ssp_stages must be >= 2");
        block_ = st_.block_size > 0 ? st_.block_size : 128;
        if (block_ % 32 || block_ > 128) return set_error(ZSME_ERR_ARG, "block_size must be a multiple of 32, <= 128");
        ZSME_CUDA(cudaSetDevice(device_));
        ZSME_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        const int C = pm_.C;
        grid_ = (C + block_ - 1) / block_;
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
        md_ = MeshDev{C, pm_.K, slot_nbr_.p, slot_meta_.p, slot_face_.p, slot_dx_.p, slot_w_.p, vol_.p,
                      rc_.p, order_.p, fn_.p, farea_.p, fc_.p, fnr_.p, pm_.F};
        opts_ = Opts{st_.reconstruction_order, st_.limiter, st_.gradient, st_.ssp_stages, st_.source};
        ZSME_CUDA(x_.alloc((size_t)NQ * C));
        ZSME_CUDA(w_.alloc((size_t)NQ * C));
        ZSME_CUDA(aux_.alloc((size_t)NA * C));
        ZSME_CUDA(fs_.alloc((size_t)pm_.K * NQ * C));
        ZSME_CUDA(tmp_a_.alloc((size_t)std::max(NQ, NA) * C));
        ZSME_CUDA(tmp_b_.alloc((size_t)std::max(NQ, NA) * C));
        ZSME_CUDA(cudaMemsetAsync(x_.p, 0, x_.n * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(aux_.p, 0, aux_.n * sizeof(double), stream_));
        // scalars: t, dt_cfl, dt_step, dt_src ; ints: active, step_idx, diag[3]
        ZSME_CUDA(scal_.alloc(4));
        ZSME_CUDA(iscal_.alloc(8));
        ZSME_CUDA(cudaMemsetAsync(scal_.p, 0, 4 * sizeof(double), stream_));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, 8 * sizeof(int), stream_));
        ZSME_CUDA(partial_.alloc(grid_));
        std::vector<double> pv(NP);
        auto dp = M::default_parameters();
        for (int i = 0; i < NP; ++i) pv[i] = params ? params[i] : dp[i];
        ZSME_CUDA(params_.upload(pv, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    StepDev step_dev(const double* dts) {
        return StepDev{scal_.p + 0, scal_.p + 1, scal_.p + 2, iscal_.p + 0, dts, iscal_.p + 1,
                       st_.t_end, st_.cfl, M::dt_max, partial_.p, grid_, iscal_.p + 2};
    }

    int set_params(const double* params) override {
        ZSME_CUDA(cudaMemcpyAsync(params_.p, params, NP * sizeof(double), cudaMemcpyHostToDevice, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    // ---------------------------------------------------------- state I/O
    int set_state(const double* q, double t, bool device) override {
        const int C = pm_.C;
        const double* src = q;
        if (!device) {
            ZSME_CUDA(cudaMemcpyAsync(tmp_a_.p, q, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, stream_));
            src = tmp_a_.p;
        }
        aos_to_soa_kernel<<<grid_, block_, 0, stream_>>>(src, x_.p, old_of_new_.p, C, NQ);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaMemsetAsync(aux_.p, 0, aux_.n * sizeof(double), stream_));
        ZSME_CUDA(cudaMemcpyAsync(scal_.p, &t, sizeof(double), cudaMemcpyHostToDevice, stream_));
        ZSME_CUDA(cudaMemsetAsync(iscal_.p, 0, 8 * sizeof(int), stream_));
        steps_ = 0;
        // constraints, then dt_start = max(ComputeTimeStep, min_dt)
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        finalize_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, sd, nullptr,
                                                             FIN_POST | FIN_WRITE | FIN_DT);
        ZSME_CUDA(cudaGetLastError());
        end_step_kernel<<<1, 256, 0, stream_>>>(sd, 0, st_.min_dt);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    int get_soa(const double* soa, int nv, double* out, bool device) {
        const int C = pm_.C;
        double* dst = device ? out : tmp_b_.p;
        soa_to_aos_kernel<<<grid_, block_, 0, stream_>>>(soa, dst, old_of_new_.p, C, nv);
        ZSME_CUDA(cudaGetLastError());
        if (!device)
            ZSME_CUDA(cudaMemcpyAsync(out, tmp_b_.p, (size_t)nv * C * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }
    int get_state(double* q, bool device) override { return get_soa(x_.p, NQ, q, device); }
    int get_aux(double* a) override { return get_soa(aux_.p, NA, a, false); }

    // ---------------------------------------------------------- pieces
    void launch_prep(const double* w, const int* active) {
        mark(ZSME_KERNEL_PREP, true);
        prep_kernel<M><<<grid_, block_, 0, stream_>>>(md_, opts_, w, aux_.p, params_.p, fs_.p, active);
        mark(ZSME_KERNEL_PREP, false);
    }
    void launch_flux(int mode, double t_host, const double* t_dev, double frac, const double* x_in, double* x_out,
                     double* base, const double* dt, const int* active) {
        mark(ZSME_KERNEL_FLUX, true);
        flux_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, opts_, fs_.p, aux_.p, params_.p, mode, t_host, t_dev,
                                                         frac, x_in, x_out, base, dt, active);
        mark(ZSME_KERNEL_FLUX, false);
    }

    int rhs(double t, const double* x_aos, double* f_aos) override {
        const int C = pm_.C;
        ZSME_CUDA(cudaMemcpyAsync(tmp_b_.p, x_aos, (size_t)NQ * C * sizeof(double), cudaMemcpyHostToDevice, stream_));
        aos_to_soa_kernel<<<grid_, block_, 0, stream_>>>(tmp_b_.p, w_.p, old_of_new_.p, C, NQ);
        launch_prep(w_.p, nullptr);
        launch_flux(MODE_RHS, t, nullptr, 0.0, nullptr, tmp_a_.p, nullptr, nullptr, nullptr);
        ZSME_CUDA(cudaGetLastError());
        return get_soa(tmp_a_.p, NQ, f_aos, false);
    }

    int update_state() override {
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        finalize_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, sd, nullptr,
                                                             FIN_PRE | FIN_WRITE);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    int source(double dt) override {
        ZSME_CUDA(cudaMemcpyAsync(scal_.p + 3, &dt, sizeof(double), cudaMemcpyHostToDevice, stream_));
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        finalize_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, sd, scal_.p + 3,
                                                             FIN_SOURCE | FIN_WRITE);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        return ZSME_OK;
    }

    int compute_dt(double* dt) override {
        StepDev sd = step_dev(nullptr);
        sd.active = nullptr;
        // a scratch CFL slot so that the resident dt is left alone
        double* keep = sd.dt_cfl;
        sd.dt_cfl = scal_.p + 3;
        finalize_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, sd, nullptr, FIN_DT);
        end_step_kernel<<<1, 256, 0, stream_>>>(sd, 0, -DBL_MAX);
        ZSME_CUDA(cudaGetLastError());
        ZSME_CUDA(cudaMemcpyAsync(dt, sd.dt_cfl, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        (void)keep;
        return ZSME_OK;
    }

    // One time step (MUSCLSolver.hpp:140-188) as a launch sequence.
    void enqueue_step(const double* dts) {
        StepDev sd = step_dev(dts);
        const double* t = sd.t;
        const double* dt = sd.dt_step;
        const int* act = sd.active;
        mark(ZSME_KERNEL_BEGIN, true);
        begin_step_kernel<<<1, 1, 0, stream_>>>(sd);
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
        mark(ZSME_KERNEL_FINALIZE, true);
        finalize_kernel<M, N><<<grid_, block_, 0, stream_>>>(md_, x_.p, aux_.p, params_.p, sd, sd.dt_step, flags);
        mark(ZSME_KERNEL_FINALIZE, false);
        mark(ZSME_KERNEL_END, true);
        end_step_kernel<<<1, 256, 0, stream_>>>(sd, 1, 0.0);
        mark(ZSME_KERNEL_END, false);
    }
    int launches_per_step() const override {
        return 3 + (st_.reconstruction_order < 2 ? 2 : 2 * st_.ssp_stages);
    }

    int step(int nsteps, const double* dts_host) override {
        if (nsteps <= 0) return ZSME_OK;
        ZSME_CUDA(cudaMemsetAsync(iscal_.p + 2, 0, 3 * sizeof(int), stream_));
        if (dts_host || profiling_) {
            // imposed dts or per-kernel timing: plain launches (the step index
            // lives on the device)
            if (dts_host) {
                ZSME_CUDA(dts_.alloc((size_t)nsteps));
                ZSME_CUDA(cudaMemcpyAsync(dts_.p, dts_host, nsteps * sizeof(double), cudaMemcpyHostToDevice, stream_));
                ZSME_CUDA(cudaMemsetAsync(iscal_.p + 1, 0, sizeof(int), stream_));
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
        steps_ += nsteps;
        return ZSME_OK;
    }

    int sync(zsme_diag* d) override {
        ZSME_CUDA(cudaStreamSynchronize(stream_));
        double sc[3];
        int is[8];
        ZSME_CUDA(cudaMemcpy(sc, scal_.p, 3 * sizeof(double), cudaMemcpyDeviceToHost));
        ZSME_CUDA(cudaMemcpy(is, iscal_.p, 8 * sizeof(int), cudaMemcpyDeviceToHost));
        if (d) {
            d->steps = is[1];
            d->time = sc[0];
            d->dt = sc[1];
            d->n_nonfinite = is[2];
            d->n_negative_depth = is[3];
            d->n_newton_unconverged = is[4];
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
