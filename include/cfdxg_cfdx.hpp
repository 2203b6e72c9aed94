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
//    same std::invalid_argument for requests the dispatch rejects;
//  * solve_poisson_mixed_gpu / solve_poisson_dirichlet_gpu -- the Poisson
//    driver of apps/poisson (core/solvers/scalar_diffusion.h:294-357) with a
//    context in front: the mesh uploaded, the cell diffusion matrix assembled
//    on the device, the pure-Neumann compatibility check and reference-cell
//    identity-row gauge, then CG with the solver's own diagonal.
#pragma once

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfdx/core/linalg/linear_solver_dispatch.h"
#include "cfdx/core/solvers/scalar_diffusion.h"
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

// A CFDX mesh on the device (the caller destroys it with cfdxg_mesh_destroy).
inline cfdxg_mesh* upload_mesh(cfdxg_context* ctx, const cfdx::core::Mesh& m) {
    const std::size_t np = m.n_points(), nf = m.n_faces(), nc = m.n_cells();
    std::vector<int64_t> fo(m.faces().offsets_data(), m.faces().offsets_data() + nf + 1);
    std::vector<int64_t> fv(m.faces().vertices_data(), m.faces().vertices_data() + fo.back());
    std::vector<int64_t> co(m.cells().offsets_data(), m.cells().offsets_data() + nc + 1);
    std::vector<int64_t> cf(m.cells().faces_data(), m.cells().faces_data() + co.back());
    std::vector<int64_t> owner(nf), neighbour(nf);
    for (std::size_t f = 0; f < nf; ++f) {
        owner[f] = static_cast<int64_t>(m.ownership().owner(f));
        neighbour[f] = m.ownership().neighbour(f) < 0 ? -1 : m.ownership().neighbour(f);
    }
    const auto& patches = m.boundary().patches();
    std::vector<int32_t> patch_of_face(nf, -1), patch_types(patches.size());
    for (std::size_t p = 0; p < patches.size(); ++p) {
        patch_types[p] = static_cast<int32_t>(patches[p].type);
        for (const auto f : patches[p].face_ids) patch_of_face[f] = static_cast<int32_t>(p);
    }
    cfdxg_mesh_desc d{};
    d.n_points = static_cast<int64_t>(np);
    d.n_faces = static_cast<int64_t>(nf);
    d.n_cells = static_cast<int64_t>(nc);
    d.px = m.points().x_data();
    d.py = m.points().y_data();
    d.pz = m.points().z_data();
    d.face_offsets = fo.data();
    d.face_vertices = fv.data();
    d.owner = owner.data();
    d.neighbour = neighbour.data();
    d.cell_offsets = co.data();
    d.cell_faces = cf.data();
    d.n_patches = static_cast<int32_t>(patches.size());
    d.patch_of_face = patch_of_face.data();
    d.patch_types = patch_types.data();
    cfdxg_mesh* mesh = nullptr;
    if (cfdxg_mesh_upload(ctx, &d, &mesh) != CFDXG_OK || cfdxg_geometry_build(ctx, mesh) != CFDXG_OK) {
        cfdxg_mesh_destroy(mesh);
        throw std::invalid_argument(cfdxg_last_error(ctx));
    }
    return mesh;
}

inline cfdx::core::ScalarDiffusionResult solve_poisson_mixed_gpu(
    cfdxg_context* ctx, const cfdx::core::Mesh& mesh, const cfdx::core::PoissonBoundaryCondition& boundary,
    const std::vector<double>& source, const cfdx::core::ScalarDiffusionConfig& config = {}) {
    using namespace cfdx::core;
    boundary.validate(mesh.n_faces());
    const std::size_t nf = mesh.n_faces(), nc = mesh.n_cells();
    if (source.size() != nc) throw std::invalid_argument("solve_poisson_mixed: source size mismatch");
    std::vector<double> bc(nf, std::numeric_limits<double>::quiet_NaN());
    std::vector<int32_t> types(nf, 0);
    for (std::size_t f = 0; f < nf; ++f) {
        if (!boundary.face_values.empty()) bc[f] = boundary.face_values[f];
        types[f] = boundary.type_for_face(f) == PoissonBoundaryType::NEUMANN ? 1 : 0;
    }
    std::unique_ptr<cfdxg_mesh, int (*)(cfdxg_mesh*)> dm(upload_mesh(ctx, mesh), cfdxg_mesh_destroy);
    cfdxg_matrix* A = nullptr;
    ScalarDiffusionResult out;
    out.rhs = Vector(nc, 0.0);
    out.solution = Vector(nc, 0.0);
    if (cfdxg_assemble_cell_diffusion(ctx, dm.get(), bc.data(), types.data(), config.diffusivity, source.data(),
                                      CFDXG_MEM_HOST, &A, out.rhs.data()) != CFDXG_OK)
        throw std::invalid_argument(cfdxg_last_error(ctx));
    std::unique_ptr<cfdxg_matrix, int (*)(cfdxg_matrix*)> hold(A, cfdxg_matrix_destroy);
    bool dirichlet = false;
    for (std::size_t f = 0; f < nf; ++f) dirichlet = dirichlet || (std::isfinite(bc[f]) && types[f] == 0);
    if (!dirichlet) {
        // pure_neumann_compatibility_residual and its scale (scalar_diffusion.h:223-238, :306-325)
        std::vector<double> fc(3 * nf), sf(3 * nf), cc(3 * nc), vol(nc);
        if (cfdxg_geometry_download(ctx, dm.get(), fc.data(), sf.data(), cc.data(), vol.data()) != CFDXG_OK)
            throw std::invalid_argument(cfdxg_last_error(ctx));
        double balance = 0.0, scale = 1.0;
        for (std::size_t c = 0; c < nc; ++c) balance += source[c] * vol[c];
        for (std::size_t c = 0; c < nc; ++c) scale += std::abs(source[c]) * vol[c];
        for (std::size_t f = 0; f < nf; ++f) {
            if (!std::isfinite(bc[f]) || types[f] != 1) continue;
            const double area = std::sqrt(sf[f] * sf[f] + sf[nf + f] * sf[nf + f] + sf[2 * nf + f] * sf[2 * nf + f]);
            balance += bc[f] * area;
            scale += std::abs(bc[f]) * area;
        }
        if (!std::isfinite(balance) || !std::isfinite(config.compatibility_tolerance) ||
            config.compatibility_tolerance < 0.0 || std::abs(balance) > config.compatibility_tolerance * scale)
            throw std::invalid_argument(
                "solve_poisson_mixed: incompatible pure-Neumann data; integral(S dV) + integral(q_n dA) must be zero");
        cfdxg_gauge* g = nullptr;
        if (cfdxg_gauge_create(ctx, A, CFDXG_GAUGE_IDENTITY_ROW, static_cast<int64_t>(config.gauge.reference_cell),
                               config.gauge.reference_value, &g) != CFDXG_OK)
            throw std::invalid_argument(cfdxg_last_error(ctx));
        std::unique_ptr<cfdxg_gauge, int (*)(cfdxg_gauge*)> gh(g, cfdxg_gauge_destroy);
        cfdxg_matrix* G = nullptr;
        Vector gauged_rhs(nc, 0.0);
        if (cfdxg_gauge_apply(ctx, g, A, out.rhs.data(), CFDXG_MEM_HOST, &G, gauged_rhs.data()) != CFDXG_OK)
            throw std::invalid_argument(cfdxg_last_error(ctx));
        hold.reset(G);
        A = G;
        out.rhs = gauged_rhs;
        out.solution(config.gauge.reference_cell) = config.gauge.reference_value;
    }
    cfdxg_request req;
    cfdxg_request_default(&req);
    req.krylov = CFDXG_KRYLOV_CG;
    req.preconditioner = CFDXG_PC_OWN_DIAGONAL;
    req.problem = CFDXG_PROBLEM_DIFFUSION;
    cfdxg_report rep{};
    const int rc = cfdxg_solve_linear_system(ctx, A, out.rhs.data(), out.solution.data(), CFDXG_MEM_HOST, &req,
                                             static_cast<int64_t>(config.max_iterations), config.tolerance, &rep);
    if (rc < 0) throw std::invalid_argument(cfdxg_last_error(ctx));
    out.linear_result.status = static_cast<SolverStatus>(rep.status);
    out.linear_result.iterations = static_cast<std::size_t>(rep.iterations);
    out.linear_result.residual = rep.residual;
    out.linear_result.residual_relative = rep.residual_relative;
    // the (gauged) system matrix, as the reference returns it
    int64_t n = 0, nnz = 0;
    cfdxg_matrix_size(A, &n, &nnz);
    std::vector<int64_t> ro(static_cast<std::size_t>(n) + 1), cols(static_cast<std::size_t>(nnz));
    std::vector<double> va(static_cast<std::size_t>(nnz));
    cfdxg_matrix_download(ctx, A, ro.data(), cols.data(), va.data());
    std::vector<SparseMatrix::Index> r32(ro.begin(), ro.end()), c32(cols.begin(), cols.end());
    out.matrix = SparseMatrix::from_sorted_csr(static_cast<std::size_t>(n), static_cast<std::size_t>(n), std::move(r32),
                                               std::move(c32), std::move(va));
    return out;
}

inline cfdx::core::ScalarDiffusionResult solve_poisson_dirichlet_gpu(
    cfdxg_context* ctx, const cfdx::core::Mesh& mesh, const cfdx::core::DirichletBoundary& boundary,
    const std::vector<double>& source, const cfdx::core::ScalarDiffusionConfig& config = {}) {
    boundary.validate(mesh.n_faces());
    for (std::size_t f = 0; f < mesh.n_faces(); ++f)
        if (!boundary.face_values.empty() && std::isfinite(boundary.face_values[f]) &&
            boundary.type_for_face(f) != cfdx::core::PoissonBoundaryType::DIRICHLET)
            throw std::invalid_argument("solve_poisson_dirichlet: all prescribed boundary faces must be Dirichlet");
    return solve_poisson_mixed_gpu(ctx, mesh, boundary, source, config);
}

}  // namespace cfdxg_cfdx
