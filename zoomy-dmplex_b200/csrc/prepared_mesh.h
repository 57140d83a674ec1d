// Model-independent host structures shared by the model translation units
// and the C ABI layer: the device-ready mesh layout and the solver interface.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "zsme.h"

namespace zsme {

// Mesh in the device layout: cells renumbered along a Hilbert curve, faces
// renumbered by their first cell, per-cell "slots" in the caller's cone order.
struct PreparedMesh {
    int dim = 2, C = 0, F = 0, K = 0;
    std::vector<int> old_of_new;           // [C] caller cell id of device cell c
    std::vector<int> new_of_old;           // [C]
    std::vector<int> slot_nbr, slot_meta, slot_face;  // [K][C]
    std::vector<double> slot_dx, slot_w;   // [K][2][C]
    std::vector<double> vol, rc;           // [C]
    std::vector<int> order;                // [C]
    std::vector<double> fn, farea, fc, fnr;  // [2][F], [F], [2][F], [2][F]
    std::vector<int> face_old_of_new;      // [F]
};

// Builds the layout (validates the connectivity; computes the least-squares
// weights as LeastSquaresGradient::Setup does, Gradient.hpp:222-298).
int prepare_mesh(const zsme_mesh& m, PreparedMesh& out);

int set_error(int code, const std::string& msg);

class SolverBase {
  public:
    virtual ~SolverBase() = default;
    virtual int n_dof_q() const = 0;
    virtual int n_dof_qaux() const = 0;
    virtual int init(PreparedMesh&& pm, const zsme_settings& st, const double* params, int device) = 0;
    virtual int set_params(const double* params) = 0;
    virtual int set_state(const double* q, double t, bool device) = 0;
    virtual int get_state(double* q, bool device) = 0;
    virtual int get_aux(double* a) = 0;
    virtual int rhs(double t, const double* x, double* f) = 0;
    virtual int update_state() = 0;
    virtual int source(double dt) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int step(int nsteps, const double* dts) = 0;
    virtual int sync(zsme_diag* d) = 0;
    virtual void* stream() = 0;
    virtual int launches_per_step() const = 0;
    virtual int set_profiling(int on) = 0;
    virtual int read_profile(double* ms, int64_t* n) = 0;
};

}  // namespace zsme
