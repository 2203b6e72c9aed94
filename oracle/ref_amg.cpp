// ref_amg.cpp -- oracle adapter: the reference's native Boomer-style AMG.
//
// TEST INFRASTRUCTURE ONLY.  Builds the reference MatrixFreeVcyclePreconditioner
// with exactly the parameters NativeAMGPreconditioner::setup passes for the
// Balanced policy (core/linalg/hypre_amg.cpp:172-219: omega 0.7, 6 pre / 6 post
// damped-Jacobi sweeps, strength 0.25, 25 levels, DirectCF interpolation, no
// constant null space, no C/F row cap, coarsening fraction 1.0) so that the
// whole hierarchy (level matrices, inverse diagonals, prolongations,
// aggregates, damping) can be exported for bit-exact comparison.  The level
// storage of that class is private; this translation unit alone re-declares
// the access specifiers so it can read it.  No reference source is modified.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "cfdx/core/linalg/amg_preconditioner.h"
#include "cfdx/core/linalg/gmres_solver.h"
#undef private
#undef protected

#include "ref_common.h"

using namespace cfdx::core;

namespace {

// Same operator as detail::OwnedSparseOperator (core/linalg/hypre_amg.cpp:13-35).
class OwnedOperator final : public LinearOperatorBase {
public:
    explicit OwnedOperator(SparseMatrix m) : matrix_(std::move(m)) {}
    std::size_t rows() const noexcept override { return matrix_.n_rows(); }
    std::size_t cols() const noexcept override { return matrix_.n_cols(); }
    void apply(const Vector& input, Vector& output) const override {
        const auto values = matrix_.matvec(input);
        if (output.size() != values.size()) output.resize(values.size());
        for (std::size_t i = 0; i < values.size(); ++i) output(i) = values[i];
    }
    SparseMatrix matrix_;
};

struct AmgHandle {
    std::unique_ptr<OwnedOperator> op;
    std::unique_ptr<MatrixFreeVcyclePreconditioner> amg;
};

}  // namespace

// constant_null_space: the flag NativeBoomerAMGPreconditioner passes through
// (hypre_amg.cpp:211-212) when the dispatch solves with NullSpaceModel::Constant.
extern "C" void* ref_amg_create_ns(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                   int32_t require_cert, int32_t constant_null_space, double* seconds) {
    try {
        auto h = std::make_unique<AmgHandle>();
        h->op = std::make_unique<OwnedOperator>(cfdx_ref::make_csr(n, ro, co, va));
        h->amg = std::make_unique<MatrixFreeVcyclePreconditioner>(
            *h->op, 0.7, 6, 6, 0.25, 25, AMGInterpolationPolicy::DirectCF, constant_null_space != 0,
            require_cert != 0, AMGSmootherPolicy::DampedJacobi, 0.0, 0, 1.0);
        const double t0 = cfdx_ref::now_seconds();
        const bool ok = h->amg->setup(h->op->matrix_);
        if (seconds) *seconds = cfdx_ref::now_seconds() - t0;
        if (!ok) {
            cfdx_ref::g_error = "AMG setup failed: " + h->amg->last_setup_error();
            return nullptr;
        }
        cfdx_ref::g_error.clear();
        return h.release();
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return nullptr;
    }
}

extern "C" void* ref_amg_create(int64_t n, const int64_t* ro, const int64_t* co,
                                const double* va, int32_t require_cert, double* seconds) {
    return ref_amg_create_ns(n, ro, co, va, require_cert, 0, seconds);
}

// Builds the reference preconditioner around an externally supplied hierarchy
// (level CSR matrices, inverse diagonals, prolongations, aggregates, damping)
// without running setup().  Used only to time the reference's own V-cycle and
// GMRES at sizes where its setup would take hours; the hierarchy must be the
// one setup() produces (the parity tests check level-by-level equality).
extern "C" void* ref_amg_create_from_levels(int32_t n_levels, const int64_t* n_rows,
                                            const int64_t* const* ro, const int64_t* const* co,
                                            const double* const* va, const double* const* inv_diag,
                                            const int64_t* const* p_off, const int64_t* const* p_col,
                                            const double* const* p_val, double omega) {
    try {
        auto h = std::make_unique<AmgHandle>();
        h->op = std::make_unique<OwnedOperator>(cfdx_ref::make_csr(n_rows[0], ro[0], co[0], va[0]));
        h->amg = std::make_unique<MatrixFreeVcyclePreconditioner>(
            *h->op, 0.7, 6, 6, 0.25, 25, AMGInterpolationPolicy::DirectCF, false, false,
            AMGSmootherPolicy::DampedJacobi, 0.0, 0, 1.0);
        auto& levels = h->amg->levels_;
        levels.resize(static_cast<std::size_t>(n_levels));
        for (int32_t l = 0; l < n_levels; ++l) {
            const int64_t n = n_rows[l];
            levels[l].A = cfdx_ref::make_csr(n, ro[l], co[l], va[l]);
            levels[l].inv_diag.assign(inv_diag[l], inv_diag[l] + n);
            if (l + 1 < n_levels) {
                levels[l].prolongation.assign(static_cast<std::size_t>(n), {});
                levels[l].aggregate.assign(static_cast<std::size_t>(n), 0);
                for (int64_t i = 0; i < n; ++i)
                    for (int64_t q = p_off[l][i]; q < p_off[l][i + 1]; ++q)
                        levels[l].prolongation[i].push_back({static_cast<std::size_t>(p_col[l][q]), p_val[l][q]});
            }
        }
        h->amg->omega_ = omega;
        cfdx_ref::g_error.clear();
        return h.release();
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return nullptr;
    }
}

// MatrixFreeVcyclePreconditioner::setup (amg_preconditioner.h:76-243) for the
// DirectCF policy with one step replaced: the C/F interpolation of each level
// (build_cf_interpolation, :1511-1885, the step whose second pass makes the
// reference's setup take hours at 10^6 rows) is read from arrays that a
// complete run of that same setup wrote out, instead of being recomputed.
// Everything else is the reference's own code in setup()'s order: the fine
// diagonal, GalerkinCSRProduct symbolic + numeric for every coarse operator
// (galerkin_csr_product.h:33-176), matrix_is_valid, build_diagonal,
// build_level_lines, and compute_stable_smoother_omega for the damping.
// coarse_rows[l] is the row count of level l (level 0 = the input matrix).
extern "C" void* ref_amg_create_from_transfers(int64_t n, const int64_t* ro, const int64_t* co,
                                               const double* va, int32_t n_levels,
                                               const int64_t* coarse_rows,
                                               const int64_t* const* p_off,
                                               const int64_t* const* p_col,
                                               const double* const* p_val,
                                               const int64_t* const* aggregate, double* seconds) {
    try {
        auto h = std::make_unique<AmgHandle>();
        h->op = std::make_unique<OwnedOperator>(cfdx_ref::make_csr(n, ro, co, va));
        h->amg = std::make_unique<MatrixFreeVcyclePreconditioner>(
            *h->op, 0.7, 6, 6, 0.25, 25, AMGInterpolationPolicy::DirectCF, false, false,
            AMGSmootherPolicy::DampedJacobi, 0.0, 0, 1.0);
        auto& P = *h->amg;
        using Level = MatrixFreeVcyclePreconditioner::Level;
        const double t0 = cfdx_ref::now_seconds();
        const auto fail = [&](const std::string& why) -> void* {
            cfdx_ref::g_error = "AMG rebuild failed: " + why;
            return nullptr;
        };
        if (n_levels < 1 || coarse_rows[0] != n) return fail("level sizes");
        P.levels_.clear();
        P.first_aggregate_.clear();
        Level fine;
        fine.A = h->op->matrix_;
        if (!MatrixFreeVcyclePreconditioner::build_diagonal(fine)) return fail("fine diagonal");
        if (!P.build_level_lines(fine)) return fail("fine lines");
        P.levels_.push_back(std::move(fine));
        for (int32_t l = 0; l + 1 < n_levels; ++l) {
            const int64_t rows = coarse_rows[l];
            if (static_cast<int64_t>(P.levels_.back().A.n_rows()) != rows) return fail("level rows");
            std::vector<MatrixFreeVcyclePreconditioner::TransferRow> prolongation(static_cast<std::size_t>(rows));
            std::vector<std::size_t> agg(static_cast<std::size_t>(rows));
            for (int64_t i = 0; i < rows; ++i) {
                for (int64_t q = p_off[l][i]; q < p_off[l][i + 1]; ++q)
                    prolongation[i].push_back({static_cast<std::size_t>(p_col[l][q]), p_val[l][q]});
                agg[i] = static_cast<std::size_t>(aggregate[l][i]);
            }
            const std::size_t coarse_n = static_cast<std::size_t>(coarse_rows[l + 1]);
            GalerkinCSRProduct product;
            SparseMatrix coarse;
            if (!product.symbolic(P.levels_.back().A, prolongation, coarse_n) ||
                !product.numeric(P.levels_.back().A, prolongation, coarse,
                                 &P.last_footprint_.galerkin_dropped_entries) ||
                !MatrixFreeVcyclePreconditioner::matrix_is_valid(coarse))
                return fail("Galerkin product at level " + std::to_string(l));
            if (P.levels_.size() == 1) P.first_aggregate_ = agg;
            Level next;
            next.A = std::move(coarse);
            if (!MatrixFreeVcyclePreconditioner::build_diagonal(next)) return fail("coarse diagonal");
            if (!P.build_level_lines(next)) return fail("coarse lines");
            P.levels_.back().aggregate = std::move(agg);
            P.levels_.back().prolongation = std::move(prolongation);
            P.levels_.back().coarse_product = std::move(product);
            P.levels_.push_back(std::move(next));
        }
        double safe_omega = 0.0;
        if (P.compute_stable_smoother_omega(P.levels_, safe_omega, &P.last_setup_error_))
            P.omega_ = safe_omega;
        else
            P.omega_ = P.configured_omega_;
        if (seconds) *seconds = cfdx_ref::now_seconds() - t0;
        cfdx_ref::g_error.clear();
        return h.release();
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return nullptr;
    }
}

// MatrixFreeVcyclePreconditioner::update_values (amg_preconditioner.h:245-314)
// on the owned operator's matrix replaced by the new values (same pattern).
extern "C" int ref_amg_update_values(void* hv, int64_t n, const int64_t* ro, const int64_t* co,
                                     const double* va) {
    try {
        auto* h = static_cast<AmgHandle*>(hv);
        h->op->matrix_ = cfdx_ref::make_csr(n, ro, co, va);
        if (!h->amg->update_values(h->op->matrix_)) {
            cfdx_ref::g_error = "AMG update_values failed";
            return 1;
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" void ref_amg_destroy(void* h) { delete static_cast<AmgHandle*>(h); }

// The cycle's constant_null_space flag on an existing handle (e.g. one built
// from supplied levels); the hierarchy itself does not depend on it.
extern "C" void ref_amg_set_constant_null_space(void* h, int32_t flag) {
    static_cast<AmgHandle*>(h)->amg->constant_null_space_ = flag != 0;
}

extern "C" int32_t ref_amg_num_levels(void* h) {
    return static_cast<int32_t>(static_cast<AmgHandle*>(h)->amg->levels_.size());
}

extern "C" double ref_amg_omega(void* h) { return static_cast<AmgHandle*>(h)->amg->omega_; }

extern "C" int ref_amg_level_sizes(void* hv, int32_t level, int64_t* n_rows, int64_t* nnz,
                                   int64_t* p_nnz) {
    auto* h = static_cast<AmgHandle*>(hv);
    const auto& L = h->amg->levels_.at(static_cast<std::size_t>(level));
    *n_rows = static_cast<int64_t>(L.A.n_rows());
    *nnz = static_cast<int64_t>(L.A.nnz());
    int64_t pn = 0;
    for (const auto& row : L.prolongation) pn += static_cast<int64_t>(row.size());
    *p_nnz = pn;
    return 0;
}

extern "C" int ref_amg_level_matrix(void* hv, int32_t level, int64_t* ro, int64_t* co,
                                    double* va, double* inv_diag) {
    auto* h = static_cast<AmgHandle*>(hv);
    const auto& L = h->amg->levels_.at(static_cast<std::size_t>(level));
    cfdx_ref::export_csr(L.A, ro, co, va);
    for (std::size_t i = 0; i < L.inv_diag.size(); ++i) inv_diag[i] = L.inv_diag[i];
    return 0;
}

extern "C" int ref_amg_level_prolongation(void* hv, int32_t level, int64_t* ro, int64_t* co,
                                          double* va, int64_t* aggregate) {
    auto* h = static_cast<AmgHandle*>(hv);
    const auto& L = h->amg->levels_.at(static_cast<std::size_t>(level));
    int64_t k = 0;
    ro[0] = 0;
    for (std::size_t i = 0; i < L.prolongation.size(); ++i) {
        for (const auto& [c, w] : L.prolongation[i]) {
            co[k] = static_cast<int64_t>(c);
            va[k] = w;
            ++k;
        }
        ro[i + 1] = k;
    }
    for (std::size_t i = 0; i < L.aggregate.size(); ++i)
        aggregate[i] = static_cast<int64_t>(L.aggregate[i]);
    return 0;
}

extern "C" int ref_amg_apply(void* hv, const double* r, double* z) {
    auto* h = static_cast<AmgHandle*>(hv);
    const std::size_t n = h->op->rows();
    Vector rv(n), zv(n);
    for (std::size_t i = 0; i < n; ++i) rv(i) = r[i];
    const bool ok = h->amg->apply(rv, zv);
    for (std::size_t i = 0; i < n; ++i) z[i] = zv(i);
    return ok ? 0 : 1;
}

// Solve phase only, on a hierarchy that was set up beforehand: the
// SparseMatrix overload of solve_gmres with setup_preconditioner = false
// (core/linalg/gmres_solver.h:690-741).
extern "C" int ref_solve_gmres_prepared(void* hv, int64_t n, const int64_t* ro,
                                        const int64_t* co, const double* va,
                                        const double* rhs, double* x, int32_t restart,
                                        int64_t max_iterations, double tolerance,
                                        ref_report_t* report) {
    try {
        auto* h = static_cast<AmgHandle*>(hv);
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n)), xv(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            b(i) = rhs[i];
            xv(i) = x[i];
        }
        const double t0 = cfdx_ref::now_seconds();
        const SolverResult r = solve_gmres(A, b, xv, restart, static_cast<std::size_t>(max_iterations),
                                           tolerance, h->amg.get(), KrylovControls{},
                                           PrecisionPolicy{}, false);
        const double t1 = cfdx_ref::now_seconds();
        for (int64_t i = 0; i < n; ++i) x[i] = xv(i);
        if (report) {
            report->status = static_cast<int32_t>(r.status);
            report->iterations = static_cast<int64_t>(r.iterations);
            report->residual = r.residual;
            report->residual_relative = r.residual_relative;
            report->physical_residual_relative = r.residual_relative;
            report->setup_seconds = 0.0;
            report->solve_seconds = t1 - t0;
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}
