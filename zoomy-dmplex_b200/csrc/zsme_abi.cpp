// C ABI of the library (include/zsme.h): model registry, argument checks,
// error reporting.  Each entry point forwards to the model's Solver with the
// handle's device current, and gives the caller's current device back on
// return, so handles on different GPUs can be used from one thread.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "prepared_mesh.h"
#include "zsme.h"

#define ZSME_MODELS(X) X(sme1d_l0_malpasset) X(sme2d_l0) X(sme2d_l1) X(sme2d_l2) X(sme2d_l4)

#define ZSME_DECLARE(NS) zsme::SolverBase* zsme_make_##NS(); void zsme_info_##NS(int* v);
ZSME_MODELS(ZSME_DECLARE)

namespace zsme {

namespace {
thread_local std::string g_err = "";

struct ModelEntry {
    const char* name;
    SolverBase* (*make)();
    void (*info)(int*);
};
#define ZSME_ENTRY(NS) ModelEntry{#NS, &zsme_make_##NS, &zsme_info_##NS},
const ModelEntry kModels[] = {ZSME_MODELS(ZSME_ENTRY)};
const int kNumModels = sizeof(kModels) / sizeof(kModels[0]);

const ModelEntry* find_model(const char* name) {
    if (!name) return nullptr;
    for (const auto& e : kModels)
        if (!std::strcmp(e.name, name)) return &e;
    return nullptr;
}
}  // namespace

int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

}  // namespace zsme

struct zsme_handle {
    zsme::SolverBase* s;
};

using zsme::set_error;

namespace {
// Makes `dev` the current device for the guard's scope and restores the
// device that was current before (cudaSetDevice is per host thread).
class DeviceGuard {
  public:
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev_) != cudaSuccess) {
            err_ = cudaGetLastError();
            return;
        }
        if (prev_ != dev) {
            err_ = cudaSetDevice(dev);
            set_ = err_ == cudaSuccess;
        }
    }
    ~DeviceGuard() {
        if (set_) cudaSetDevice(prev_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
    int check() const {
        if (err_ == cudaSuccess) return ZSME_OK;
        return set_error(ZSME_ERR_CUDA, std::string("selecting the handle's device: ") + cudaGetErrorString(err_));
    }

  private:
    int prev_ = 0;
    bool set_ = false;
    cudaError_t err_ = cudaSuccess;
};
}  // namespace

// a valid handle, with its device current until the entry point returns
#define CHECK_H(h)                                                          \
    if (!(h) || !(h)->s) return set_error(ZSME_ERR_ARG, "null handle");     \
    DeviceGuard dev_guard_((h)->s->device());                               \
    if (int dev_rc_ = dev_guard_.check()) return dev_rc_
// calls that address "the" state need a single-instance handle
#define CHECK_SINGLE(h)                                                                          \
    CHECK_H(h);                                                                                  \
    if ((h)->s->n_instances() != 1)                                                              \
    return set_error(ZSME_ERR_ARG, "batch handle: use the zsme_batch_* state functions")

extern "C" {

const char* zsme_version(void) { return "zsme 0.1 (sm_100a, FP64)"; }
const char* zsme_last_error(void) { return zsme::g_err.c_str(); }
int zsme_num_models(void) { return zsme::kNumModels; }
const char* zsme_model_name(int i) { return (i >= 0 && i < zsme::kNumModels) ? zsme::kModels[i].name : nullptr; }

int zsme_model_info(const char* model, int32_t* nq, int32_t* na, int32_t* np, int32_t* dim) {
    const auto* e = zsme::find_model(model);
    if (!e) return set_error(ZSME_ERR_MODEL, std::string("unknown model: ") + (model ? model : "(null)"));
    int v[4];
    e->info(v);
    if (nq) *nq = v[0];
    if (na) *na = v[1];
    if (np) *np = v[2];
    if (dim) *dim = v[3];
    return ZSME_OK;
}

int zsme_create(const char* model, const zsme_mesh* mesh, const zsme_settings* settings, const double* params,
                int device, zsme_handle** out) {
    if (!out || !mesh || !settings) return set_error(ZSME_ERR_ARG, "null argument");
    *out = nullptr;
    const auto* e = zsme::find_model(model);
    if (!e) return set_error(ZSME_ERR_MODEL, std::string("unknown model: ") + (model ? model : "(null)"));
    if (settings->reconstruction_order < 1 || settings->reconstruction_order > 2)
        return set_error(ZSME_ERR_ARG, "reconstruction_order must be 1 or 2");
    if (!(settings->cfl > 0)) return set_error(ZSME_ERR_ARG, "cfl must be > 0");
    if (settings->positivity < ZSME_POSITIVITY_NONE || settings->positivity > ZSME_POSITIVITY_MOOD)
        return set_error(ZSME_ERR_ARG, "positivity must be ZSME_POSITIVITY_NONE, _ZHANG_SHU or _MOOD");
    zsme::PreparedMesh pm;
    int rc = zsme::prepare_mesh(*mesh, pm);
    if (rc) return rc;
    DeviceGuard dev_guard(device);
    if ((rc = dev_guard.check())) return rc;
    zsme::SolverBase* s = e->make();
    rc = s->init(std::move(pm), *settings, params, device);
    if (rc) {
        delete s;
        return rc;
    }
    *out = new zsme_handle{s};
    return ZSME_OK;
}

int zsme_mesh_tiles(const zsme_mesh* mesh, int32_t tile_faces, int32_t* stats) {
    if (!mesh || !stats) return set_error(ZSME_ERR_ARG, "null argument");
    zsme::PreparedMesh pm;
    int rc = zsme::prepare_mesh(*mesh, pm);
    if (rc) return rc;
    zsme::FaceTiles t;
    rc = zsme::build_tiles(pm, tile_faces, t);
    if (rc) return rc;
    int64_t covered = 0, slots = 0;
    for (int c = 0; c < pm.C; ++c)
        for (int j = 0; j < pm.K; ++j) slots += t.ord_lf[(size_t)j * pm.C + c] >= 0;
    for (int b = 0; b < t.n; ++b) covered += t.face_off[b + 1] - t.face_off[b];
    stats[0] = t.n;
    stats[1] = t.max_faces;
    stats[2] = (int32_t)t.in_faces.size();
    stats[3] = (int32_t)covered;
    stats[4] = (int32_t)slots;
    return ZSME_OK;
}

int zsme_destroy(zsme_handle* h) {
    if (!h) return ZSME_OK;
    if (h->s) {
        DeviceGuard dev_guard(h->s->device());
        delete h->s;
    }
    delete h;
    return ZSME_OK;
}

int zsme_set_state(zsme_handle* h, const double* q, double t) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null state");
    return h->s->set_state(0, q, t, false);
}
int zsme_set_state_device(zsme_handle* h, const double* q, double t) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null state");
    return h->s->set_state(0, q, t, true);
}
int zsme_get_state(zsme_handle* h, double* q) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->get_state(0, q, false);
}
int zsme_get_state_device(zsme_handle* h, double* q) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->get_state(0, q, true);
}
int zsme_get_cells(zsme_handle* h, int32_t n, const int32_t* cells, double* q, int32_t on_device) {
    CHECK_SINGLE(h);
    if (n > 0 && (!cells || !q)) return set_error(ZSME_ERR_ARG, "null cell list or state");
    return h->s->get_cells(n, cells, q, on_device != 0);
}
int zsme_set_cells(zsme_handle* h, int32_t n, const int32_t* cells, const double* q, int32_t on_device) {
    CHECK_SINGLE(h);
    if (n > 0 && (!cells || !q)) return set_error(ZSME_ERR_ARG, "null cell list or state");
    return h->s->set_cells(n, cells, q, on_device != 0);
}
int zsme_set_state_async(zsme_handle* h, const double* q, double t) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null state");
    return h->s->set_state_async(q, t);
}
int zsme_get_state_async(zsme_handle* h, double* q) {
    CHECK_SINGLE(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->get_state_async(q);
}
int zsme_stream_wait_copies(zsme_handle* h) {
    CHECK_SINGLE(h);
    return h->s->stream_wait_copies();
}
int zsme_get_aux(zsme_handle* h, double* a) {
    CHECK_SINGLE(h);
    if (!a) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->get_aux(0, a);
}
int zsme_rhs(zsme_handle* h, double t, const double* x, double* f) {
    CHECK_H(h);
    if (!x || !f) return set_error(ZSME_ERR_ARG, "null buffer");
    return h->s->rhs(t, x, f);
}
int zsme_implicit_function(zsme_handle* h, double t, const double* x, const double* xdot, double* f) {
    CHECK_SINGLE(h);
    if (!x || !xdot || !f) return set_error(ZSME_ERR_ARG, "null buffer");
    return h->s->implicit_function(t, x, xdot, f);
}
int zsme_implicit_jacobian(zsme_handle* h, double t, const double* x, double shift, double* diag, double* faces) {
    CHECK_SINGLE(h);
    if (!x) return set_error(ZSME_ERR_ARG, "null buffer");
    return h->s->implicit_jacobian(t, x, shift, diag, faces);
}
int zsme_implicit_stats(zsme_handle* h, int32_t* stats) {
    CHECK_SINGLE(h);
    if (!stats) return set_error(ZSME_ERR_ARG, "null output");
    int v[4];
    int rc = h->s->implicit_stats(v);
    for (int i = 0; i < 4; ++i) stats[i] = v[i];
    return rc;
}
int zsme_update_state(zsme_handle* h) {
    CHECK_H(h);
    return h->s->update_state();
}
int zsme_source(zsme_handle* h, double dt) {
    CHECK_H(h);
    return h->s->source(dt);
}
int zsme_compute_dt(zsme_handle* h, double* dt) {
    CHECK_H(h);
    if (!dt) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->compute_dt(0, dt);
}
int zsme_step(zsme_handle* h, int32_t n) {
    CHECK_H(h);
    if (n < 0) return set_error(ZSME_ERR_ARG, "negative step count");
    return h->s->step(n, nullptr);
}
int zsme_step_dt(zsme_handle* h, int32_t n, const double* dts) {
    CHECK_H(h);
    if (n < 0 || (n > 0 && !dts)) return set_error(ZSME_ERR_ARG, "bad dts");
    for (int i = 0; i < n; ++i)
        if (!(dts[i] >= 0)) return set_error(ZSME_ERR_ARG, "dts must be >= 0");
    return h->s->step(n, dts);
}
int zsme_step_dt_device(zsme_handle* h, int32_t n, const double* d_dts) {
    CHECK_SINGLE(h);
    if (n < 0 || (n > 0 && !d_dts)) return set_error(ZSME_ERR_ARG, "bad dts");
    return h->s->step_device_dts(n, d_dts);
}
int zsme_get_time_device(zsme_handle* h, double* d_t, double* d_dt) {
    CHECK_SINGLE(h);
    return h->s->get_time_device(d_t, d_dt);
}
int zsme_get_diag(zsme_handle* h, zsme_diag* d) {
    CHECK_H(h);
    if (!d) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->sync(0, d);
}
int zsme_sync(zsme_handle* h) {
    CHECK_H(h);
    zsme_diag d;
    int rc = h->s->sync(0, &d);
    if (rc) return rc;
    if (d.n_nonfinite > 0 || d.n_negative_depth > 0)
        return set_error(ZSME_ERR_STATE, "state check: " + std::to_string(d.n_nonfinite) + " non-finite, " +
                                             std::to_string(d.n_negative_depth) + " negative-depth cell updates");
    return ZSME_OK;
}
int zsme_get_time(zsme_handle* h, double* t, double* dt) {
    CHECK_H(h);
    zsme_diag d;
    int rc = h->s->sync(0, &d);
    if (rc) return rc;
    if (t) *t = d.time;
    if (dt) *dt = d.dt;
    return ZSME_OK;
}
int zsme_set_params(zsme_handle* h, const double* p) {
    CHECK_H(h);
    if (!p) return set_error(ZSME_ERR_ARG, "null params");
    return h->s->set_params(p);
}
void* zsme_stream(zsme_handle* h) { return (h && h->s) ? h->s->stream() : nullptr; }
int zsme_device(zsme_handle* h, int32_t* device) {
    if (!h || !h->s) return set_error(ZSME_ERR_ARG, "null handle");
    if (device) *device = h->s->device();
    return ZSME_OK;
}
int zsme_launches_per_step(zsme_handle* h, int32_t* n) {
    CHECK_H(h);
    if (n) *n = h->s->launches_per_step();
    return ZSME_OK;
}

int zsme_set_profiling(zsme_handle* h, int enable) {
    CHECK_H(h);
    return h->s->set_profiling(enable);
}
int zsme_read_profile(zsme_handle* h, double* ms, int64_t* n) {
    CHECK_H(h);
    return h->s->read_profile(ms, n);
}

int zsme_batch_create(const char* model, int32_t n, const zsme_mesh* meshes, const zsme_settings* settings,
                      const double* params, int device, zsme_handle** out) {
    if (!out || !meshes || !settings || n <= 0) return set_error(ZSME_ERR_ARG, "null argument or empty batch");
    *out = nullptr;
    const auto* e = zsme::find_model(model);
    if (!e) return set_error(ZSME_ERR_MODEL, std::string("unknown model: ") + (model ? model : "(null)"));
    if (settings->reconstruction_order < 1 || settings->reconstruction_order > 2)
        return set_error(ZSME_ERR_ARG, "reconstruction_order must be 1 or 2");
    if (!(settings->cfl > 0)) return set_error(ZSME_ERR_ARG, "cfl must be > 0");
    if (settings->positivity < ZSME_POSITIVITY_NONE || settings->positivity > ZSME_POSITIVITY_MOOD)
        return set_error(ZSME_ERR_ARG, "positivity must be ZSME_POSITIVITY_NONE, _ZHANG_SHU or _MOOD");
    std::vector<zsme::PreparedMesh> parts(n);
    for (int i = 0; i < n; ++i) {
        int rc = zsme::prepare_mesh(meshes[i], parts[i]);
        if (rc) return set_error(rc, "instance " + std::to_string(i) + ": " + zsme_last_error());
    }
    zsme::PreparedMesh pm;
    int rc = zsme::concat_meshes(parts, pm);
    if (rc) return rc;
    DeviceGuard dev_guard(device);
    if ((rc = dev_guard.check())) return rc;
    zsme::SolverBase* s = e->make();
    rc = s->init(std::move(pm), *settings, params, device);
    if (rc) {
        delete s;
        return rc;
    }
    *out = new zsme_handle{s};
    return ZSME_OK;
}
int zsme_batch_size(zsme_handle* h, int32_t* n) {
    CHECK_H(h);
    if (n) *n = h->s->n_instances();
    return ZSME_OK;
}
int zsme_batch_set_state(zsme_handle* h, int32_t i, const double* q, double t) {
    CHECK_H(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null state");
    return h->s->set_state(i, q, t, false);
}
int zsme_batch_get_state(zsme_handle* h, int32_t i, double* q) {
    CHECK_H(h);
    if (!q) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->get_state(i, q, false);
}
int zsme_batch_get_time(zsme_handle* h, int32_t i, double* t, double* dt) {
    CHECK_H(h);
    zsme_diag d;
    int rc = h->s->sync(i, &d);
    if (rc) return rc;
    if (t) *t = d.time;
    if (dt) *dt = d.dt;
    return ZSME_OK;
}
int zsme_set_launch(zsme_handle* h, const int32_t* blocks) {
    CHECK_H(h);
    if (!blocks) return set_error(ZSME_ERR_ARG, "null block sizes");
    return h->s->set_launch(
        zsme::LaunchConfig{blocks[0], blocks[1], blocks[2], blocks[3], blocks[4], blocks[5], blocks[6], blocks[7],
                           blocks[8], blocks[9]});
}
int zsme_adjoint(zsme_handle* h, int32_t nsteps, int32_t checkpoint_every, int32_t n_obs, const int32_t* obs_step,
                 const int32_t* obs_cell, const int32_t* obs_comp, const double* obs_target,
                 const double* obs_weight, double* loss, double* grad_q_aos, double* grad_params, double* dts) {
    CHECK_SINGLE(h);
    zsme::AdjointSpec a;
    a.nsteps = nsteps;
    a.every = checkpoint_every;
    a.nobs = n_obs;
    a.obs_step = obs_step;
    a.obs_cell = obs_cell;
    a.obs_comp = obs_comp;
    a.obs_target = obs_target;
    a.obs_weight = obs_weight;
    return h->s->adjoint(a, loss, grad_q_aos, grad_params, dts);
}
int zsme_adjoint_phases(zsme_handle* h, double* ms3) {
    CHECK_SINGLE(h);
    if (!ms3) return set_error(ZSME_ERR_ARG, "null output");
    return h->s->adjoint_phases(ms3);
}
int zsme_adjoint_overlapped(zsme_handle* h, int32_t* overlapped) {
    CHECK_SINGLE(h);
    if (!overlapped) return set_error(ZSME_ERR_ARG, "null output");
    *overlapped = h->s->adjoint_overlapped() ? 1 : 0;
    return ZSME_OK;
}
int zsme_get_launch(zsme_handle* h, int32_t* blocks) {
    CHECK_H(h);
    if (!blocks) return set_error(ZSME_ERR_ARG, "null output");
    const zsme::LaunchConfig lc = h->s->launch();
    blocks[0] = lc.prep;
    blocks[1] = lc.face;
    blocks[2] = lc.gather;
    blocks[3] = lc.finalize;
    blocks[4] = lc.prep_occ;
    blocks[5] = lc.face_occ;
    blocks[6] = lc.finalize_occ;
    blocks[7] = lc.tile_faces;
    blocks[8] = lc.fuse_final;
    blocks[9] = lc.prep_lean;
    return ZSME_OK;
}

}  // extern "C"
