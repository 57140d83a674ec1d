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
// Several independent instances (an ensemble) are concatenated cell- and
// face-wise; old_of_new then holds instance-local caller ids.
struct PreparedMesh {
    int dim = 2, C = 0, F = 0, K = 0;
    std::vector<int> old_of_new;           // [C] caller cell id of device cell c (within its instance)
    std::vector<int> new_of_old;           // [C] (single instance only)
    std::vector<int> slot_nbr, slot_meta, slot_face;  // [K][C]
    std::vector<double> slot_dx, slot_w;   // [K][2][C]
    std::vector<double> vol, rc;           // [C]
    std::vector<int> order;                // [C]
    std::vector<double> fn, farea, fc, fnr;  // [2][F], [F], [2][F], [2][F]
    std::vector<int> face_old_of_new;      // [F]
    std::vector<int> face_L, face_R, face_bc;  // [F] support (new cell ids) and marker
    int n_inst = 1;
    std::vector<int> inst_cell_off, inst_face_off;  // [n_inst + 1]
    std::vector<int> cell_inst, face_inst;          // [C], [F] (n_inst > 1 only)
};

// Block sizes of the kernels (the autotuner's knobs).
struct LaunchConfig {
    int prep, face, gather, finalize;  // threads per block
    int prep_occ = 1, face_occ = 1;    // register cap, blocks per SM: prep 1, 2, 3, 4, 6, 8; face 1-4
    int finalize_occ = 1;              // register cap of finalize, blocks of 128 per SM: 1-4
    int tile_faces = 0;                // > 0: fused face + gather kernel over tiles of at most this many
                                       // faces (64..1024); 0: separate face and gather kernels
    int fuse_final = 0;                // 1: with separate face and gather kernels, the last stage's
                                       // gather runs inside the finalize kernel
    int prep_lean = 1;                 // order-2 face states: prep_kernel (0), prep_lean_kernel (1),
                                       // prep_split_kernel with 2..4 threads per cell
};

// Tiles of the fused face + gather kernel.  A tile is a run of consecutive
// cells; it evaluates the faces whose lowest cell lies in the tile (a
// contiguous range, faces being sorted by their lowest cell) and the
// "incoming" faces whose other cell lies in an earlier tile, keeps their
// contributions in shared memory and sums them per cell.  An incoming face is
// evaluated by both tiles it touches, each keeping its own side.
struct FaceTiles {
    int n = 0;          // tiles
    int max_faces = 0;  // most faces evaluated by one tile (shared memory rows)
    std::vector<int> cell_off, face_off, in_off;  // [n + 1]
    std::vector<int> in_faces;                    // [in_off[n]] incoming faces, tile by tile
    // [K][C]: the cell's j-th face in accumulation order (increasing original
    // face id) as (local face index << 1) | (cell is support[0]); -1: no face
    // or an exterior face without a condition (no flux)
    std::vector<int> ord_lf;
};
int build_tiles(const PreparedMesh& p, int max_faces, FaceTiles& out);

// Builds the layout (validates the connectivity; computes the least-squares
// weights as LeastSquaresGradient::Setup does, Gradient.hpp:222-298).
int prepare_mesh(const zsme_mesh& m, PreparedMesh& out);
// Concatenates prepared instances (same dim and K) into one layout.
int concat_meshes(std::vector<PreparedMesh>& parts, PreparedMesh& out);

int set_error(int code, const std::string& msg);

// Least-squares observations of a discrete adjoint run (zsme_adjoint):
// loss = sum_j weight_j (Q_{step_j}[cell_j, comp_j] - target_j)^2.
struct AdjointSpec {
    int nsteps = 0, every = 1, nobs = 0;
    const int* obs_step = nullptr;
    const int* obs_cell = nullptr;   // caller cell ids
    const int* obs_comp = nullptr;
    const double* obs_target = nullptr;
    const double* obs_weight = nullptr;  // nullptr: all 1
};

class SolverBase {
  public:
    virtual ~SolverBase() = default;
    virtual int n_dof_q() const = 0;
    virtual int n_dof_qaux() const = 0;
    virtual int n_instances() const = 0;
    // the CUDA device the handle's buffers and stream live on
    virtual int device() const = 0;
    virtual int init(PreparedMesh&& pm, const zsme_settings& st, const double* params, int device) = 0;
    virtual int set_params(const double* params) = 0;
    virtual int set_state(int inst, const double* q, double t, bool device) = 0;
    virtual int get_state(int inst, double* q, bool device) = 0;
    virtual int get_cells(int n, const int* cells, double* q, bool device) = 0;
    virtual int set_cells(int n, const int* cells, const double* q, bool device) = 0;
    virtual int set_state_async(const double* q, double t) = 0;
    virtual int get_state_async(double* q) = 0;
    virtual int stream_wait_copies() = 0;
    virtual int get_aux(int inst, double* a) = 0;
    virtual int rhs(double t, const double* x, double* f) = 0;
    virtual int update_state() = 0;
    virtual int source(double dt) = 0;
    virtual int compute_dt(int inst, double* dt) = 0;
    virtual int step(int nsteps, const double* dts) = 0;
    // imposed dts read from device memory, in stream order (no host synchronisation)
    virtual int step_device_dts(int nsteps, const double* d_dts) = 0;
    // time and CFL dt of instance 0 copied to device memory, in stream order
    virtual int get_time_device(double* d_t, double* d_dt) = 0;
    virtual int sync(int inst, zsme_diag* d) = 0;
    virtual void* stream() = 0;
    virtual int launches_per_step() const = 0;
    virtual int set_profiling(int on) = 0;
    virtual int read_profile(double* ms, int64_t* n) = 0;
    virtual int set_launch(const LaunchConfig& lc) = 0;
    virtual LaunchConfig launch() const = 0;
    // loss, gradient with respect to the state at call time (caller order, AoS),
    // gradient with respect to the parameters, and the dt of every step
    virtual int adjoint(const AdjointSpec& spec, double* loss, double* grad_q, double* grad_params,
                        double* dts) = 0;
    // device times of the last adjoint call's forward pass, replays and reverse sweep (ms)
    virtual int adjoint_phases(double* ms) = 0;
    virtual bool adjoint_overlapped() const = 0;
    virtual int implicit_function(double t, const double* x_aos, const double* xdot_aos, double* f_aos) = 0;
    virtual int implicit_jacobian(double t, const double* x_aos, double a, double* diag, double* offdiag) = 0;
    virtual int implicit_stats(int* out) const = 0;
};

}  // namespace zsme
