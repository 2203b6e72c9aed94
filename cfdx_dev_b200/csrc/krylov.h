// krylov.h -- device-resident GMRES / FGMRES (see krylov.cu).
#pragma once
#include <functional>
#include <limits>

#include "objects.h"

namespace cfdxg {

// core/linalg/krylov_controls.h:10-26
struct KrylovControls {
    int restart_min = 10;
    int restart_max = 512;
    bool adaptive_restart = true;
    int64_t residual_replacement_period = 50;
    bool residual_replacement = true;
    double residual_replacement_gap_ratio = 10.0;
    double target_reduction_per_cycle = 0.1;
    // Two passes of classical instead of modified Gram-Schmidt: the same
    // projections, formed as h = V^T w and w -= V h (two passes over the basis
    // per pass instead of 2(j+1)); not the reference's order of operations.
    bool classical_gram_schmidt = false;
};

// core/linalg/solver_status.h:45-72
struct KrylovResult {
    int status = CFDXG_NOT_APPLICABLE;
    int64_t iterations = 0;
    double residual = 0.0;
    double residual_relative = 0.0;
    int64_t residual_replacements = 0;
    double max_true_recursive_gap = 0.0;
    double min_true_recursive_ratio = std::numeric_limits<double>::infinity();
    double max_true_recursive_ratio = 0.0;
    double max_true_residual = 0.0;
    double min_true_residual = std::numeric_limits<double>::infinity();
    int64_t first_residual_replacement = 0;
    int64_t last_residual_replacement = 0;
    int64_t preconditioner_applications = 0;
};

// Enqueues z = M^-1 v on the context stream (device vectors); returns false
// when it cannot run.  Non-finite results are reported through the status word.
// z = M v for the j-th Arnoldi vector of the current restart cycle (j = 0: the
// normalised true residual the cycle starts from).
using RightPreconditioner = std::function<bool(const double* v, double* z, int j)>;

// Called after every Arnoldi step with the Givens estimate of the residual norm.
using IterationObserver = std::function<void(double estimated_residual)>;

// projection: 0, or the entry e of the normalised constant null-space vector,
// every operator application and preconditioner action then being projected
// (P A P and P M P, P v = v - (v . e) e).
KrylovResult gmres_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x,
                         int restart, int64_t max_iter, double tolerance, const RightPreconditioner* pc,
                         const KrylovControls& controls, const IterationObserver* observer = nullptr,
                         double projection = 0.0);

// The constant null space (core/linalg/null_space.h, projected_gmres.h).
// Every entry of NullSpaceProjector::constant(n)'s normalised basis vector.
double constant_null_space_entry(int64_t n);
// is_compatible(b), is_null_space(A) and is_bilateral_null_space(A), their
// norms taken on the device (scaled two-pass norms instead of hypot sums).
struct NullSpaceChecks {
    bool compatible = false, null_space = false, bilateral = false;
    double component = 0.0, operator_residual = 0.0;
};
NullSpaceChecks null_space_checks(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b);
// solve_projected_gmres (projected_gmres.h:84-150); `setup`, when given, runs
// after the early-exit check, and a false return makes the solve NOT_APPLICABLE.
KrylovResult projected_gmres_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x,
                                   int restart, int64_t max_iter, double tolerance, const RightPreconditioner* pc,
                                   const KrylovControls& controls, const IterationObserver* observer,
                                   const std::function<bool()>* setup);

// core/linalg/cg_solver.h:45-560 with a preconditioner object (pc, its j
// argument unused); `setup`, when given, runs after the initial-residual
// check as the reference's setup_preconditioner and a false return makes the
// solve NOT_APPLICABLE.  own_diagonal: pc divides by the matrix diagonal and
// the solve follows the solver's own-diagonal branch (no preconditioner
// object, the legacy solve_cg overload, cg_solver.h:591-603) -- its residual
// replacement rule instead of the adaptive one.
// null_space: the projected CG of solve_cg(..., NullSpaceProjector) -- a
// compatible b and A e = 0 or NOT_APPLICABLE, then x, the initial residual,
// every z, A p, x and r after the update, the replaced residuals and every
// search direction projected (cg_solver.h:74-79, 93, 149, 203, 262, 295-298,
// 376, 517, 558).
KrylovResult cg_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x, int64_t max_iter,
                      double tolerance, const RightPreconditioner& pc, const std::function<bool()>* setup,
                      bool own_diagonal = false, bool null_space = false);

// Scaled two-pass 2-norm of a device vector (krylov_norm2).
double device_norm2(cfdxg_context* ctx, const cfdxg_matrix* A, const double* a);
// Enqueues out = sum_i a_i b_i (deterministic fixed-order reduction) into a device scalar.
void enqueue_dot(cfdxg_context* ctx, int64_t n, const double* a, const double* b, double* out);
// ||b - A x|| with the FP64 operator.
double device_residual_norm(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, const double* x);

}  // namespace cfdxg
