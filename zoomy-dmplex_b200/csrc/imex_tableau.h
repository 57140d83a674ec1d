// Butcher tableau of the additive Runge-Kutta scheme "2E" that the reference's
// IMEX strategy selects (PETSc TSARKIMEX type "2e", SolverStrategies.hpp:62-85):
// three stages, second order; the explicit part (transport) has an explicit
// first stage, the implicit part (source) is an L-stable singly diagonally
// implicit scheme with diagonal gamma = 1 - 1/sqrt(2) after an explicit first
// stage; the weights b are the implicit part's last row for both parts.
// Shared by the GPU kernels and the CPU restatement, so both round the same
// constants (folded at compile time in IEEE double).
#pragma once

namespace zsme {
namespace ark2e {
constexpr double s2 = 1.414213562373095048802;
constexpr double gamma = 1.0 - 1.0 / s2;
// explicit part A[i][j] (j < i)
constexpr double a10 = 2.0 - s2;
constexpr double a20 = (3.0 - 2.0 * s2) / 6.0;
constexpr double a21 = (3.0 + 2.0 * s2) / 6.0;
// implicit part At[i][j] (j <= i)
constexpr double t10 = gamma;
constexpr double t20 = 1.0 / (2.0 * s2);
constexpr double t21 = 1.0 / (2.0 * s2);
// weights (both parts) and the stage times c_i (t0 + c_i dt)
constexpr double b0 = 1.0 / (2.0 * s2);
constexpr double b1 = 1.0 / (2.0 * s2);
constexpr double b2 = gamma;
constexpr double c1 = 2.0 - s2;
constexpr double c2 = 1.0;
// the implicit source of a stage is skipped in cells drier than this depth,
// and its Jacobian there is the identity block (ModularSolver.hpp:101-104,
// 428-436)
constexpr double dry_residual = 1e-6;
constexpr double dry_jacobian = 1e-4;
}  // namespace ark2e
}  // namespace zsme
