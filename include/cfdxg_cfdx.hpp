// cfdxg_cfdx.hpp -- CFDX-side adapters over the C ABI (header-only C++).
//
// Compiled inside CFDX, with its sources (src/) and this directory on the
// include path and libcfdxg.so linked:
//
//  * GpuNativeAMGPreconditioner -- a cfdx::core::Preconditioner
//    (core/linalg/preconditioner.h:18-28) whose setup, update_values and
//    apply run the library's native AMG (the reference's hierarchy, bit for
//    bit) with its V-cycle on the GPU; make_scalar_preconditioner
//    (core/linalg/linear_solver_dispatch.h:169-225) can return it for
//    PreconditionerModel::NativeAMG when a GPU context is configured, and the
//    reference's own CPU Krylov solvers then call it unchanged;
//  * solve_linear_system_gpu -- the signature of solve_linear_system
//    (linear_solver_dispatch.h:227-234) with a context in front, routed
//    through cfdxg_solve_linear_system: the whole Krylov solve on the device,
//    the same automatic plan, scaling and FP64 physical certificate, and the
//    same std::invalid_argument for requests the dispatch rejects.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfdx/core/linalg/linear_solver_dispatch.h"
#include "cfdxg.h"

namespace cfdxg_cfdx {

// A device copy of a finalized CFDX CSR matrix (the caller destroys it).
inline cfdxg_matrix* upload(cfdxg_context* ctx, const cfdx::core::SparseMatrix& A) {
    const std::vector<int64_t> ro(A.row_offsets_data(), A.row_offsets_data() + A.n_rows() + 1);
    const std::vector<int64_t> co(A.columns_data(), A.columns_data() + A.nnz());
    cfdxg_matrix* M = nullptr;
    if (cfdxg_matrix_create(ctx, static_cast<int64_t>(A.n_rows()), ro.data(), co.data(), A.values_data(),
                            CFDXG_MEM_HOST, &M) != CFDXG_OK)
        return nullptr;
    return M;
}

class GpuNativeAMGPreconditioner final : public cfdx::core::Preconditioner {
public:
    explicit GpuNativeAMGPreconditioner(cfdxg_context* ctx, int32_t precision = CFDXG_PRECISION_FP64,
                                        bool require_smoother_certificate = false)
        : ctx_(ctx) {
        cfdxg_amg_options o;
        cfdxg_amg_options_default(&o);
        o.precision = precision;
        o.require_smoother_certificate = require_smoother_certificate ? 1 : 0;
        if (cfdxg_amg_create(ctx_, &o, &amg_) != CFDXG_OK) throw std::runtime_error("cfdxg_amg_create failed");
    }
    ~GpuNativeAMGPreconditioner() override {
        cfdxg_matrix_destroy(A_);
        cfdxg_amg_destroy(amg_);
    }
    GpuNativeAMGPreconditioner(const GpuNativeAMGPreconditioner&) = delete;
    GpuNativeAMGPreconditioner& operator=(const GpuNativeAMGPreconditioner&) = delete;

    bool setup(const cfdx::core::SparseMatrix& A) override {
        replace(A);
        return A_ && cfdxg_amg_setup(ctx_, amg_, A_) == CFDXG_OK;
    }
    // The reference's numeric refresh, on the device; false when the pruned
    // coarse pattern changed (the caller then sets up again).
    bool update_values(const cfdx::core::SparseMatrix& A) override {
        replace(A);
        return A_ && cfdxg_amg_update_values(ctx_, amg_, A_) == CFDXG_OK;
    }
    bool apply(const cfdx::core::Vector& r, cfdx::core::Vector& z) const override {
        if (z.size() != r.size()) z.resize(r.size());
        return cfdxg_amg_apply(ctx_, amg_, r.data(), z.data(), CFDXG_MEM_HOST) == CFDXG_OK;
    }
    const char* name() const override { return cfdxg_amg_name(amg_); }
    const char* last_error() const { return cfdxg_amg_last_error(amg_); }

private:
    void replace(const cfdx::core::SparseMatrix& A) {
        cfdxg_matrix_destroy(A_);
        A_ = upload(ctx_, A);
    }
    cfdxg_context* ctx_;
    cfdxg_amg* amg_ = nullptr;
    cfdxg_matrix* A_ = nullptr;
};

inline cfdx::core::LinearSolveReport solve_linear_system_gpu(
    cfdxg_context* ctx, const cfdx::core::SparseMatrix& matrix, const cfdx::core::Vector& rhs,
    cfdx::core::Vector& solution, cfdx::core::LinearProblemKind problem,
    const cfdx::core::LinearSolverRequest& request = {}, std::size_t max_iterations = 1000,
    double tolerance = 1e-12, int32_t precision = CFDXG_PRECISION_FP64) {
    using namespace cfdx::core;
    LinearSolveReport report;
    if (request.null_space != NullSpaceModel::None)
        throw std::invalid_argument("a projected null space is not provided by libcfdxg");
    if (matrix.n_rows() != matrix.n_cols() || rhs.size() != matrix.n_rows() || solution.size() != matrix.n_rows()) {
        report.result.status = SolverStatus::NOT_APPLICABLE;
        return report;
    }
    cfdxg_request req;
    cfdxg_request_default(&req);
    req.krylov = static_cast<int32_t>(request.krylov);
    req.preconditioner = static_cast<int32_t>(request.preconditioner);
    req.gmres_restart = request.gmres_restart;
    req.problem = static_cast<int32_t>(problem);
    req.scaling = static_cast<int32_t>(request.scaling);
    req.precision = precision;
    cfdxg_matrix* A = upload(ctx, matrix);
    if (!A) throw std::invalid_argument(cfdxg_last_error(ctx));
    cfdxg_report rep{};
    const int rc = cfdxg_solve_linear_system(ctx, A, rhs.data(), solution.data(), CFDXG_MEM_HOST, &req,
                                             static_cast<int64_t>(max_iterations), tolerance, &rep);
    cfdxg_matrix_destroy(A);
    if (rc < 0) throw std::invalid_argument(cfdxg_last_error(ctx));
    report.result.status = static_cast<SolverStatus>(rep.status);
    report.result.iterations = static_cast<std::size_t>(rep.iterations);
    report.result.residual = rep.residual;
    report.result.residual_relative = rep.residual_relative;
    report.result.residual_replacements = static_cast<std::size_t>(rep.residual_replacements);
    report.result.max_true_recursive_gap = rep.max_true_recursive_gap;
    report.physical_residual_relative = rep.physical_residual_relative;
    report.applied_scaling = request.scaling;
    report.plan.problem = problem;
    report.plan.krylov = static_cast<KrylovModel>(rep.plan_krylov);
    report.plan.preconditioner = rep.plan_preconditioner == CFDXG_PC_OWN_DIAGONAL
                                     ? PreconditionerModel::None
                                     : static_cast<PreconditionerModel>(rep.plan_preconditioner);
    report.plan.automatic_krylov = request.krylov == KrylovModel::Auto;
    report.plan.automatic_preconditioner = request.preconditioner == PreconditionerModel::Auto;
    report.plan.reason = cfdxg_plan_reason(ctx);
    if (report.result.status == SolverStatus::NOT_APPLICABLE) report.preconditioner_error = cfdxg_last_error(ctx);
    return report;
}

}  // namespace cfdxg_cfdx
