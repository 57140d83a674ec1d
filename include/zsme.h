/*
 * zsme.h -- C ABI of the B200 shallow-water-moment (SME) time step.
 *
 * The entry points replace the hot-path calls of the reference's
 * MUSCLSolver driver (reference file:line cited on each declaration):
 *   TransportStep::FormRHS          (TransportStep.hpp:325)  -> zsme_rhs
 *   TransportStep::UpdateState      (TransportStep.hpp:196)  -> zsme_update_state
 *   SourceStep::Solve               (SourceStep.hpp:72)      -> zsme_source
 *   VirtualSolver::ComputeTimeStep  (VirtualSolver.hpp:285)  -> zsme_compute_dt
 *   MUSCLSolver::Run step loop      (MUSCLSolver.hpp:140-188)-> zsme_step
 *
 * Conventions (mirroring PETSc's): every function returns an int status,
 * ZSME_OK (0) on success; on failure zsme_last_error() describes it.  The
 * caller owns host buffers; the library owns device buffers.  A handle is
 * single-threaded and stream-ordered (one CUDA stream per handle).  A handle
 * lives on the device given to zsme_create; every call on it makes that
 * device current for the call's duration and restores the calling thread's
 * current device before returning, so handles on several GPUs may be driven
 * from one thread in any order.  States
 * cross the boundary cell-major/interleaved ("AoS", [n_cells][n_dof_q], the
 * layout of the reference's PETSc Vec with block size n_dof_q) in the
 * caller's cell order; inside, the library renumbers cells along a Hilbert
 * curve and stores every variable as its own FP64 array.
 */
#ifndef ZSME_H
#define ZSME_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZSME_OK 0
#define ZSME_ERR_ARG 1      /* invalid argument (null pointer, size, name) */
#define ZSME_ERR_CUDA 2     /* a CUDA call failed; message has the CUDA error */
#define ZSME_ERR_MODEL 3    /* unknown model name */
#define ZSME_ERR_STATE 4    /* non-finite state or negative depth detected */
#define ZSME_ERR_MESH 5     /* inconsistent mesh connectivity */
#define ZSME_ERR_LIMIT 6    /* a compiled size limit was exceeded */
#define ZSME_ERR_SOLVE 7    /* an implicit step's Newton iteration did not converge; the state, time and
                               step history are those before the step */

/* Face boundary markers in zsme_mesh.face_bc */
#define ZSME_FACE_INTERIOR (-1)
#define ZSME_FACE_NO_CONDITION (-2)  /* exterior face whose tag has no BC: no flux */

/*
 * Cell-centred finite-volume mesh: the quantities the reference takes from
 * DMPlexGetGeometryFVM and the DMPlex cone/support (TransportStep.hpp:388-410).
 * Coordinates are always 2 doubles per point (y = 0 for 1-D meshes).
 */
typedef struct zsme_mesh {
    int32_t dim;                  /* 1 or 2; must equal the model's dimension */
    int32_t n_cells;
    int32_t n_faces;
    int32_t max_faces;            /* K: faces per cell (2 for 1-D, 3 triangles) */
    const double* cell_centroid;  /* [n_cells][2] */
    const double* cell_volume;    /* [n_cells] */
    const int32_t* cell_faces;    /* [n_cells][K] cone order, -1 padded */
    const int32_t* face_cells;    /* [n_faces][2] support; [1] = -1 on the boundary */
    const double* face_centroid;  /* [n_faces][2] */
    const double* face_normal;    /* [n_faces][2] area-weighted, support[0] -> support[1] */
    const int32_t* face_bc;       /* [n_faces] ZSME_FACE_INTERIOR, bc index >= 0, or
                                     ZSME_FACE_NO_CONDITION */
    const uint8_t* cell_cfl_skip; /* [n_cells] nonzero: the cell does not constrain the CFL dt
                                     (the halo cells of a mesh partition); NULL: none */
} zsme_mesh;

#define ZSME_LIMITER_NONE 0       /* settings.solver.limiter == "none" */
#define ZSME_LIMITER_TVD 1        /* VacuumLimiter + TVDLimiter (Reconstruction.hpp:170-175) */
#define ZSME_GRADIENT_GREEN_GAUSS 0 /* GreenGaussGradient (Gradient.hpp:43-191) */
#define ZSME_GRADIENT_LSQ 1       /* LeastSquaresGradient (Gradient.hpp:196-360) */
/* settings.solver.positivity (Settings.hpp:24-27, ModularSolver.hpp:46-58) */
#define ZSME_POSITIVITY_NONE 0      /* "none": LinearReconstructor with Vacuum + TVD limiting */
#define ZSME_POSITIVITY_ZHANG_SHU 1 /* "zhang_shu": eta-well-balanced reconstruction, Venkatakrishnan
                                       slopes and the Zhang-Shu theta (TransportStep.hpp:241-323,
                                       Reconstruction.hpp:247-287); order 2 clamps CFL to 1/6
                                       (MUSCLSolver.hpp:33-38) */
#define ZSME_POSITIVITY_MOOD 2      /* "mood": the same reconstruction without theta, and cells whose
                                       depth ends below -1e-10 redone by a first-order Euler step
                                       (MUSCLSolver.hpp:130-171, 197-229) */

/* settings.solver.time_integration (Settings.hpp:34, MUSCLSolver.hpp:56-72) */
#define ZSME_TIME_SPLITTING 0 /* "splitting": SSP-RK(s,2) transport, then the implicit source step */
#define ZSME_TIME_IMEX 1      /* "imex": additive Runge-Kutta 2E (explicit transport, implicit source per
                                 cell; SolverStrategies.hpp:62-128) at the step's CFL dt */
#define ZSME_TIME_IMPLICIT 2  /* "implicit": BDF (order 1 on the first step after a state is set, 2
                                 after) of F = Xdot - S(X) - R(X), Newton with a matrix-free Jacobian
                                 and GMRES preconditioned by the diagonal blocks of the reference's
                                 assembled Jacobian (SolverStrategies.hpp:133-195) at the step's CFL
                                 dt; single-instance handles, positivity "none" or "zhang_shu" */

/* The solver keys of the reference's Settings (Settings.hpp:13-40) that change
 * the step. */
typedef struct zsme_settings {
    double cfl;                   /* solver.cfl */
    double t_end;                 /* solver.t_end */
    double min_dt;                /* solver.min_dt (floor of the first dt only) */
    int32_t reconstruction_order; /* 1: PCM + forward Euler; 2: linear + SSP-RK(s,2) */
    int32_t limiter;              /* ZSME_LIMITER_* */
    int32_t gradient;             /* ZSME_GRADIENT_* */
    int32_t ssp_stages;           /* s of SSP-RK(s,2), >= 2 */
    int32_t source;               /* 1: operator-split implicit source ("splitting") */
    int32_t block_size;           /* CUDA block size, 0 = library default */
    int32_t positivity;           /* ZSME_POSITIVITY_* */
    int32_t refresh_derivative_aux; /* solver.refresh_derivative_aux: before every state update, fill the
                                     plugin's derivative aux slots (its field-level update_aux_variables;
                                     Green-Gauss derivatives, TransportStep.hpp:161-192) */
    int32_t time_integration;     /* ZSME_TIME_SPLITTING, ZSME_TIME_IMEX or ZSME_TIME_IMPLICIT */
    int32_t reserved[3];
    double wet_dry_eps;           /* solver.wet_dry_eps (reference default 1e-2): dry threshold of the
                                     positivity variants, read only when positivity != NONE */
} zsme_settings;

/* Health counters of the last step (failure detection without faulting). */
typedef struct zsme_diag {
    int64_t steps;                /* steps taken since zsme_set_state */
    double time;                  /* simulated time */
    double dt;                    /* dt of the next step (CFL) */
    int32_t n_nonfinite;          /* cells with a non-finite value */
    int32_t n_negative_depth;     /* cells with h < -1e-10 (MUSCLSolver.hpp:206) */
    int32_t n_newton_unconverged; /* cells whose Newton hit 15 iterations */
    int32_t n_mood_cells;         /* cells redone at first order by MOOD (ZSME_POSITIVITY_MOOD) */
    int32_t n_newton_deferred;    /* cell updates whose Newton solve left the register fast path for the
                                     full pivoted elimination (summed over the last zsme_step call) */
} zsme_diag;

typedef struct zsme_handle zsme_handle;

/* Library version string. */
const char* zsme_version(void);
/* Message of the last failed call on this thread (never NULL). */
const char* zsme_last_error(void);
/* Number of compiled models and their names (e.g. "sme2d_l2"). */
int zsme_num_models(void);
const char* zsme_model_name(int i);
/* Model constants: n_dof_q, n_dof_qaux, n_parameters, dimension. */
int zsme_model_info(const char* model, int32_t* n_dof_q, int32_t* n_dof_qaux,
                    int32_t* n_parameters, int32_t* dimension);

/* Build a solver for `model` on `mesh` (VirtualSolver::SetupArchitecture,
 * VirtualSolver.hpp:386-525; ModularSolver::InitializeComponents,
 * ModularSolver.hpp:39-76; LeastSquaresGradient::Setup, Gradient.hpp:222-298).
 * params: n_parameters doubles, or NULL for the model defaults. */
int zsme_create(const char* model, const zsme_mesh* mesh, const zsme_settings* settings,
                const double* params, int device, zsme_handle** out);
int zsme_destroy(zsme_handle* h);
/* Host-only inspection of the tiling the fused face + gather kernel uses for
 * `mesh` at tile_faces (see zsme_set_launch); no device is touched.  No
 * counterpart in the reference.  stats[5]: tiles, most faces evaluated by a
 * tile, incoming faces (faces evaluated a second time by the tile of their
 * higher cell), faces covered by the tiles' own ranges (= n_faces), and the
 * cell-face incidences that carry a flux. */
int zsme_mesh_tiles(const zsme_mesh* mesh, int32_t tile_faces, int32_t* stats);

/* Load Q (host, AoS, caller order) as the state at time t, apply the physical
 * constraints and compute the first dt = max(ComputeTimeStep, min_dt)
 * (MUSCLSolver.hpp:51-54,103). */
int zsme_set_state(zsme_handle* h, const double* q_aos, double t);
/* Copy the state / aux state out (host, AoS, caller order). */
int zsme_get_state(zsme_handle* h, double* q_aos);
int zsme_get_aux(zsme_handle* h, double* a_aos);
/* Same with device pointers (zero-copy from torch), caller order. */
int zsme_set_state_device(zsme_handle* h, const double* d_q_aos, double t);
int zsme_get_state_device(zsme_handle* h, double* d_q_aos);
/* Asynchronous forms of zsme_set_state / zsme_get_state for pipelined calls
 * (single-instance handles; no counterpart in the reference, whose state
 * stays in host memory).  They return at once.  The copies run on two copy
 * streams of the handle, one per direction, through double-buffered device
 * staging, ordered against the handle's stream.  A read-back can therefore
 * overlap the next state's upload and the steps in between.  With
 * page-locked host buffers (cudaHostAlloc / cudaHostRegister) the copies
 * are truly asynchronous.  The caller keeps q_aos unchanged, and does not
 * read the output buffer, until zsme_sync (which waits for the copies too)
 * has returned.  Two reads in a row must go to different host buffers if
 * the first is read before zsme_sync.  zsme_stream_wait_copies makes the
 * handle's stream wait (on the device) for every copy issued so far, e.g.
 * before recording a timing event on zsme_stream.  The staging buffers
 * (4 x n_cells x n_dof_q doubles) are allocated by the first call. */
/* The state of n selected cells (caller ids; single-instance handles), for
 * the halo exchange of a partitioned mesh (no counterpart in the reference,
 * where PETSc's ghost-point scatters do this): q_aos [n][n_dof_q].  With
 * on_device the cell list and q_aos are device pointers, else host.
 * zsme_set_cells also recomputes those cells' aux variables; time, dt and
 * the other cells are left alone. */
int zsme_get_cells(zsme_handle* h, int32_t n, const int32_t* cells, double* q_aos, int32_t on_device);
int zsme_set_cells(zsme_handle* h, int32_t n, const int32_t* cells, const double* q_aos, int32_t on_device);
int zsme_set_state_async(zsme_handle* h, const double* q_aos, double t);
int zsme_get_state_async(zsme_handle* h, double* q_aos);
int zsme_stream_wait_copies(zsme_handle* h);

/* F = dQ/dt of the transport for state X (TransportStep::FormRHS,
 * TransportStep.hpp:325-357).  Host AoS buffers, caller order. */
int zsme_rhs(zsme_handle* h, double t, const double* x_aos, double* f_aos);
/* The fully implicit strategy's residual F(t, X, Xdot) = Xdot - S(X) - R(X)
 * (SolverStrategies.hpp:163-174 IFunctionWrapper: S the source at the
 * clamped state, zero where the depth is below 1e-6, R = FormRHS).  Host AoS
 * buffers [C][n_dof_q], caller order.  Needs time_integration
 * ZSME_TIME_IMPLICIT and a single-instance handle. */
int zsme_implicit_function(zsme_handle* h, double t, const double* x_aos, const double* xdot_aos, double* f_aos);
/* The preconditioning matrix of the implicit strategy at (t, X, shift a)
 * (ModularSolver::FormImplicitJacobian, ModularSolver.hpp:238-371): per cell
 * a I - dS/dQ - dS/dAux dAux/dQ (a I where the clamped depth is below 1e-4)
 * plus each face's forward-difference flux and fluctuation Jacobians at the
 * cell states scaled by area / volume.  diag_blocks [C][n_dof_q][n_dof_q] in
 * caller cell order (row-major blocks); face_blocks [F][2][n_dof_q][n_dof_q]
 * per caller face: the block at (row cell face_cells[0], column
 * face_cells[1]) and the one at (row face_cells[1], column face_cells[0]),
 * zero for boundary faces.  Either pointer may be NULL. */
int zsme_implicit_jacobian(zsme_handle* h, double t, const double* x_aos, double shift, double* diag_blocks,
                           double* face_blocks);
/* Counters of the last implicit step: Newton iterations, GMRES iterations
 * (all Newton iterations), line-search halvings, and how Newton stopped (1:
 * residual norm within tolerance, 2: update below 1e-8 of the state, 0:
 * neither within 50 iterations). */
int zsme_implicit_stats(zsme_handle* h, int32_t* stats4);
/* Physical constraints on the resident state (MUSCLSolver.hpp:234-254):
 * update_variables clamp + update_aux_variables (TransportStep.hpp:196-230). */
int zsme_update_state(zsme_handle* h);
/* Implicit per-cell source over dt on the resident state
 * (SourceStep::Solve, SourceStep.hpp:72-122). */
int zsme_source(zsme_handle* h, double dt);
/* CFL time step of the resident state (VirtualSolver.hpp:285-357). */
int zsme_compute_dt(zsme_handle* h, double* dt);

/* Advance nsteps steps of the MUSCLSolver loop (MUSCLSolver.hpp:140-188):
 * dt clamped to land on t_end, SSP-RK(s,2) transport, constraints, implicit
 * source, constraints, CFL dt.  Steps after t_end are no-ops.  Runs on the
 * device without host synchronisation (one CUDA graph per step). */
int zsme_step(zsme_handle* h, int32_t nsteps);
/* Same, but with the dt of every step imposed by the caller (dts[nsteps]). */
int zsme_step_dt(zsme_handle* h, int32_t nsteps, const double* dts);
/* Same, with the dts in device memory (d_dts[nsteps]), read in stream order:
 * a distributed caller can reduce the parts' CFL dts on the device (an
 * all-reduce with MIN, the reference's MPI_Allreduce of VirtualSolver.hpp:349)
 * and step without synchronising the host.  Single-instance handles. */
int zsme_step_dt_device(zsme_handle* h, int32_t nsteps, const double* d_dts);
/* The time and the CFL dt of the next step copied to device memory (d_t,
 * d_dt; either may be NULL) in stream order, without synchronising the host.
 * Single-instance handles. */
int zsme_get_time_device(zsme_handle* h, double* d_t, double* d_dt);
/* Wait for the handle's stream; returns ZSME_ERR_STATE if the last step left
 * non-finite values or negative depth (counts in zsme_diag). */
int zsme_sync(zsme_handle* h);
int zsme_get_diag(zsme_handle* h, zsme_diag* out);
int zsme_get_time(zsme_handle* h, double* t, double* dt);
int zsme_set_params(zsme_handle* h, const double* params);
/* The CUDA stream (cudaStream_t) the handle launches on. */
void* zsme_stream(zsme_handle* h);
/* The CUDA device ordinal the handle lives on (zsme_create's `device`). */
int zsme_device(zsme_handle* h, int32_t* device);
/* Kernel launches of one zsme_step step. */
int zsme_launches_per_step(zsme_handle* h, int32_t* n);

/* Per-kernel CUDA-event timing.  While enabled, zsme_step launches without
 * the CUDA graph, brackets every kernel with events on the handle's stream
 * and, at the end of each call, accumulates the durations per kind. */
#define ZSME_KERNEL_BEGIN 0     /* begin_step: dt clamp to t_end */
#define ZSME_KERNEL_PREP 1      /* clamp + bounds + gradient + face states */
#define ZSME_KERNEL_FLUX 2      /* face fluxes, each face once */
#define ZSME_KERNEL_FINALIZE 3  /* constraints + source + CFL partials */
#define ZSME_KERNEL_END 4       /* dt reduction + time advance */
#define ZSME_KERNEL_GATHER 5    /* per-cell sum of face contributions + stage update */
#define ZSME_KERNEL_FALLBACK 6  /* finalize of the cells whose Newton update needs the full-size GEPP */
#define ZSME_KERNEL_MOOD 7      /* MOOD first-order override (ZSME_POSITIVITY_MOOD) */
#define ZSME_KERNEL_KINDS 8
int zsme_set_profiling(zsme_handle* h, int enable);
/* ms[ZSME_KERNEL_KINDS]: summed milliseconds; n[...]: launches. */
int zsme_read_profile(zsme_handle* h, double* ms, int64_t* n);

/* Ensembles.  No counterpart in the reference, which advances one mesh per
 * run (MUSCLSolver::Run, MUSCLSolver.hpp:22-194); here n independent
 * instances (own mesh, parameters, time and CFL dt) share one handle and
 * every kernel launch of zsme_step advances all of them.  meshes[n];
 * params: n * n_parameters doubles or NULL.  zsme_step / zsme_update_state /
 * zsme_source act on all instances; states move per instance. */
int zsme_batch_create(const char* model, int32_t n, const zsme_mesh* meshes, const zsme_settings* settings,
                      const double* params, int device, zsme_handle** out);
int zsme_batch_size(zsme_handle* h, int32_t* n);
int zsme_batch_set_state(zsme_handle* h, int32_t i, const double* q_aos, double t);
int zsme_batch_get_state(zsme_handle* h, int32_t i, double* q_aos);
int zsme_batch_get_time(zsme_handle* h, int32_t i, double* t, double* dt);

/* Launch configuration, 10 ints: threads per block {prep, face, gather,
 * finalize} (multiples of 32, <= 128), the register caps {prep, face,
 * finalize} as resident blocks of 128 threads per SM (1 = uncapped; prep 2,
 * 3, 4, 6 or 8, face and finalize 2..4), tile_faces: 0 runs the face
 * fluxes and the per-cell gather as two kernels with the face contributions
 * in device memory; 64..1024 runs them as one kernel over tiles of
 * consecutive cells evaluating at most that many faces each, the
 * contributions kept in shared memory (the face block size and cap apply);
 * fuse_final: 1 lets the finalize kernel form the last SSP stage's result
 * itself from the face contributions (separate face and gather kernels,
 * order 2, positivity other than "mood"), so that result never round-trips
 * through device memory; prep_lean: 1 (default) forms the order-2 face
 * states with the lean kernel (32-bit offsets, branch-free neighbour
 * bounds), 0 with the plain one, 2..4 with the lean kernel split over that
 * many threads per cell, each owning a slice of the components (blocks of
 * 64 or 96..128 threads of its own; the prep block size does not apply and
 * its register cap takes 4, 6, 8 or none).  Every configuration gives the
 * same results bit for bit.
 * The knobs of the autotuner (zoomy-dmplex_b200/autotune.py).  Setting them
 * outside stream capture only: a new tile_faces rebuilds the tiles. */
int zsme_set_launch(zsme_handle* h, const int32_t* blocks);
int zsme_get_launch(zsme_handle* h, int32_t* blocks);

/* Discrete adjoint of nsteps steps from the resident state (single-instance
 * handle).  No counterpart in the reference, which has no derivative path;
 * it differentiates the zsme_step loop (MUSCLSolver.hpp:140-188) as
 * written: the TVD limiter's branches, the clamps of update_variables and
 * the implicit Newton source (SourceStep.hpp:125-209, by the implicit-
 * function theorem at its converged state) included, with the CFL dt of each
 * step recorded by the forward run and held fixed.
 * Loss: sum_j w_j (Q_{obs_step[j]}[obs_cell[j], obs_comp[j]] - obs_target[j])^2,
 * Q_k the state after k steps (0 = the resident state), cells in caller
 * order; obs_weight may be NULL (all 1).  The forward run keeps a checkpoint
 * every checkpoint_every steps and the reverse pass recomputes each segment.
 * Outputs (host, any may be NULL): *loss; grad_q_aos [n_cells][n_dof_q], the
 * gradient with respect to the resident state (its component 0 is the
 * gradient with respect to the bathymetry b); grad_params [n_parameters];
 * dts [nsteps], the dt sequence used.  The handle ends holding the state
 * after nsteps steps, as zsme_step(h, nsteps) would leave it. */
int zsme_adjoint(zsme_handle* h, int32_t nsteps, int32_t checkpoint_every, int32_t n_obs,
                 const int32_t* obs_step, const int32_t* obs_cell, const int32_t* obs_comp,
                 const double* obs_target, const double* obs_weight, double* loss, double* grad_q_aos,
                 double* grad_params, double* dts);
/* Device time (ms) of the last zsme_adjoint call's three phases: the
 * forward run with checkpoints, the segment replays into the tape, and the
 * reverse sweep.  When the call overlapped its replays with the reverse
 * sweep (zsme_adjoint_overlapped), the second figure is the first replay
 * alone (the one nothing overlaps) and the third the rest of the reverse
 * phase, replays included; the sum of the two is the reverse phase's device
 * time either way.  No counterpart in the reference. */
int zsme_adjoint_phases(zsme_handle* h, double* ms3);
/* 1 when the last zsme_adjoint call replayed each checkpoint segment on a
 * side stream into a second tape buffer while the reverse sweep of the
 * segment after it ran (every segment full, at least two, and device memory
 * for both tapes), else 0.  The gradients are the same bit for bit either
 * way.  No counterpart in the reference. */
int zsme_adjoint_overlapped(zsme_handle* h, int32_t* overlapped);

/* CFL time step of a caller-owned state with no device allocation.
 * No counterpart in the reference, which has no GPU path.  It serves callers
 * that cannot allocate device memory at the moment they need a step (a host
 * code that reserves its device memory up front and forbids allocation
 * afterwards, or one running under a fixed memory budget): instead of
 * cudaMalloc it uses a 512 KB scratch array compiled into the library, which
 * every GPU that loads the library holds until the process exits.
 * All pointers are device pointers, cells in any order (the same in all
 * arrays): d_q_aos [n_cells][n_dof_q], d_aux_aos [n_cells][n_dof_qaux],
 * d_rc [n_cells] (min over the cell's faces of |x_c - x_f|; a cell whose
 * d_rc is >= DBL_MAX, +inf included, is left out of the minimum -- the way
 * a partitioned caller keeps its halo cells out of the CFL dt), d_params
 * [n_parameters]; dt (cfl * min r_c/lambda_c, or the model's dt_max) is
 * written to *d_dt in stream order on `stream` (a cudaStream_t; NULL = the
 * default stream).  n_cells > ZSME_NOALLOC_MAX_CELLS returns ZSME_ERR_LIMIT.
 * The first call on a device (and in each CUDA context on it) looks the
 * scratch address up and must come before any stream capture on that
 * device.  All calls share the scratch: calls that overlap on the GPU race. */
#define ZSME_NOALLOC_MAX_CELLS (1 << 24)
int zsme_compute_dt_noalloc(const char* model, int32_t n_cells, const double* d_q_aos,
                            const double* d_aux_aos, const double* d_rc, const double* d_params,
                            double cfl, double* d_dt, void* stream);

/* Measured FP64 rate of GPU `device`, for the FP64 roofline of the step's
 * arithmetic-bound kernels.  No counterpart in the reference.  Runs
 * independent chains of fused multiply-adds on every SM for a few
 * milliseconds and writes the best of five timed launches, counting two
 * flops per FMA, to *tflops (TFLOP/s).  The step's kernels compile without
 * FMA contraction and issue one add or multiply per instruction, so half of
 * this rate bounds them. */
int zsme_fp64_fma_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* ZSME_H */
