// ref_linalg.cpp -- oracle adapter: reference geometry cache, Poisson
// assembly, solve_linear_system dispatch and mesh fixtures.
//
// TEST INFRASTRUCTURE ONLY (see ref_abi.h).  Every function forwards to the
// reference's own implementation compiled from its sources.
#include "cfdx/core/geometry/geometry_cache.h"
#include "cfdx/core/linalg/linear_solver_dispatch.h"
#include "cfdx/core/linalg/linear_system_capture.h"
#include "cfdx/core/solvers/scalar_diffusion.h"
#include "validation/radiation_tetrahedral_mesh_v52.h"

#include "ref_common.h"

#include <cstring>

using namespace cfdx::core;

extern "C" const char* ref_last_error(void) { return cfdx_ref::g_error.c_str(); }

extern "C" int ref_fixture_tet_v52_sizes(int64_t n, int64_t* sizes) {
    try {
        const Mesh m = cfdx::testing::radiation_v52::tetrahedral_mesh(static_cast<std::size_t>(n));
        sizes[0] = static_cast<int64_t>(m.n_points());
        sizes[1] = static_cast<int64_t>(m.n_faces());
        sizes[2] = static_cast<int64_t>(m.faces().n_vertices());
        sizes[3] = static_cast<int64_t>(m.n_cells());
        sizes[4] = static_cast<int64_t>(m.cells().offsets_data()[m.n_cells()]);
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int ref_fixture_tet_v52(int64_t n, double* px, double* py, double* pz,
                                   int64_t* fo, int64_t* fv, int64_t* owner, int64_t* neighbour,
                                   int64_t* co, int64_t* cf) {
    try {
        const Mesh m = cfdx::testing::radiation_v52::tetrahedral_mesh(static_cast<std::size_t>(n));
        for (std::size_t i = 0; i < m.n_points(); ++i) {
            px[i] = m.points().x(i);
            py[i] = m.points().y(i);
            pz[i] = m.points().z(i);
        }
        for (std::size_t f = 0; f <= m.n_faces(); ++f) fo[f] = static_cast<int64_t>(m.faces().offsets_data()[f]);
        for (std::size_t k = 0; k < m.faces().n_vertices(); ++k) fv[k] = static_cast<int64_t>(m.faces().vertices_data()[k]);
        for (std::size_t f = 0; f < m.n_faces(); ++f) {
            owner[f] = static_cast<int64_t>(m.ownership().owner(f));
            neighbour[f] = m.ownership().neighbour(f);
        }
        for (std::size_t c = 0; c <= m.n_cells(); ++c) co[c] = static_cast<int64_t>(m.cells().offsets_data()[c]);
        for (std::size_t k = 0; k < m.cells().offsets_data()[m.n_cells()]; ++k)
            cf[k] = static_cast<int64_t>(m.cells().faces_data()[k]);
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

static void export_vec3(const std::vector<Vec3>& v, double* out) {
    const std::size_t n = v.size();
    for (std::size_t i = 0; i < n; ++i) {
        out[i] = v[i].x;
        out[n + i] = v[i].y;
        out[2 * n + i] = v[i].z;
    }
}

extern "C" int ref_geometry_cache(const ref_mesh_t* m, double* fc, double* sf, double* cc, double* cv) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        const GeometryCache g = make_geometry_cache(mesh);
        export_vec3(g.face_centres, fc);
        export_vec3(g.face_Sf, sf);
        export_vec3(g.cell_centres, cc);
        for (std::size_t c = 0; c < g.cell_volumes.size(); ++c) cv[c] = g.cell_volumes[c];
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int64_t ref_assemble_diffusion(const ref_mesh_t* m, const double* bc, double gamma,
                                          const double* source, int64_t* ro, int64_t* co,
                                          double* va, double* rhs, double* seconds) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        DirichletBoundary boundary = PoissonBoundaryCondition::dirichlet(mesh.n_faces());
        for (std::size_t f = 0; f < mesh.n_faces(); ++f) boundary.face_values[f] = bc[f];
        const std::vector<double> src(source, source + m->n_cells);
        Vector b;
        const GeometryCache geometry = make_geometry_cache(mesh);
        const double t0 = cfdx_ref::now_seconds();
        const SparseMatrix A = assemble_cell_diffusion_matrix(mesh, boundary, gamma, src, b, geometry);
        if (seconds) *seconds = cfdx_ref::now_seconds() - t0;
        for (std::size_t i = 0; i < b.size(); ++i) rhs[i] = b(i);
        return cfdx_ref::export_csr(A, ro, co, va);
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int ref_solve_linear_system(int64_t n, const int64_t* ro, const int64_t* co,
                                       const double* va, const double* rhs, double* x,
                                       int32_t krylov, int32_t preconditioner, int32_t restart,
                                       int64_t max_iterations, double tolerance,
                                       ref_report_t* report) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n)), xv(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            b(i) = rhs[i];
            xv(i) = x[i];
        }
        LinearSolverRequest request;
        request.krylov = static_cast<KrylovModel>(krylov);
        request.preconditioner = static_cast<PreconditionerModel>(preconditioner);
        request.gmres_restart = restart;
        const double t0 = cfdx_ref::now_seconds();
        const LinearSolveReport r = solve_linear_system(
            A, b, xv, LinearProblemKind::PressurePoisson, request,
            static_cast<std::size_t>(max_iterations), tolerance);
        const double t1 = cfdx_ref::now_seconds();
        for (int64_t i = 0; i < n; ++i) x[i] = xv(i);
        if (report) {
            report->status = static_cast<int32_t>(r.result.status);
            report->iterations = static_cast<int64_t>(r.result.iterations);
            report->residual = r.result.residual;
            report->residual_relative = r.result.residual_relative;
            report->physical_residual_relative = r.physical_residual_relative;
            report->setup_seconds = 0.0;
            report->solve_seconds = t1 - t0;
        }
        cfdx_ref::g_error = r.preconditioner_error;
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// solve_linear_system with the request's null-space model
// (LinearSolverRequest::null_space, linear_solver_dispatch.h:360-400): with
// NullSpaceModel::Constant the dispatch builds the native AMG with a constant
// null space and runs solve_projected_gmres (projected_gmres.h:84-155) or the
// projected CG (cg_solver.h:45-650).
extern "C" int ref_solve_linear_system_ns(int64_t n, const int64_t* ro, const int64_t* co,
                                          const double* va, const double* rhs, double* x,
                                          int32_t krylov, int32_t preconditioner, int32_t restart,
                                          int64_t max_iterations, double tolerance, int32_t null_space,
                                          ref_report_t* report) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n)), xv(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            b(i) = rhs[i];
            xv(i) = x[i];
        }
        LinearSolverRequest request;
        request.krylov = static_cast<KrylovModel>(krylov);
        request.preconditioner = static_cast<PreconditionerModel>(preconditioner);
        request.gmres_restart = restart;
        request.null_space = static_cast<NullSpaceModel>(null_space);
        const LinearSolveReport r = solve_linear_system(
            A, b, xv, LinearProblemKind::PressurePoisson, request,
            static_cast<std::size_t>(max_iterations), tolerance);
        for (int64_t i = 0; i < n; ++i) x[i] = xv(i);
        if (report) {
            report->status = static_cast<int32_t>(r.result.status);
            report->iterations = static_cast<int64_t>(r.result.iterations);
            report->residual = r.result.residual;
            report->residual_relative = r.result.residual_relative;
            report->physical_residual_relative = r.physical_residual_relative;
            report->setup_seconds = 0.0;
            report->solve_seconds = 0.0;
        }
        cfdx_ref::g_error = r.preconditioner_error;
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int ref_spmv(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                        const double* x, double* y) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        const std::vector<double> xv(x, x + n);
        const auto yv = A.matvec(xv);
        for (int64_t i = 0; i < n; ++i) y[i] = yv[i];
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/linear_system_capture.h:170  write_linear_system_capture
extern "C" int ref_write_capture(const char* path, int64_t n, const int64_t* ro, const int64_t* co,
                                 const double* va, const double* rhs, const double* guess, int32_t problem,
                                 int32_t null_space, int32_t scaling, int64_t max_iterations, double tolerance) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n)), x(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            b(i) = rhs[i];
            x(i) = guess[i];
        }
        write_linear_system_capture(path, A, b, x, static_cast<LinearProblemKind>(problem),
                                    static_cast<NullSpaceModel>(null_space),
                                    static_cast<LinearScalingModel>(scaling),
                                    static_cast<std::size_t>(max_iterations), tolerance);
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/linear_system_capture.h:233  read_linear_system_capture: sizes
// and metadata (n, nnz, problem, null_space, scaling, max_iterations) into
// meta[6] and the tolerance into *tolerance, then the arrays when given.
extern "C" int ref_read_capture(const char* path, int64_t* meta, double* tolerance, int64_t* ro, int64_t* co,
                                double* va, double* rhs, double* guess) {
    try {
        const LinearSystemCapture c = read_linear_system_capture(path);
        const std::size_t n = c.matrix.n_rows(), nnz = c.matrix.nnz();
        meta[0] = static_cast<int64_t>(n);
        meta[1] = static_cast<int64_t>(nnz);
        meta[2] = static_cast<int64_t>(c.problem);
        meta[3] = static_cast<int64_t>(c.null_space);
        meta[4] = static_cast<int64_t>(c.scaling);
        meta[5] = static_cast<int64_t>(c.max_iterations);
        *tolerance = c.tolerance;
        if (ro) {
            for (std::size_t i = 0; i <= n; ++i) ro[i] = c.matrix.row_offsets_data()[i];
            for (std::size_t k = 0; k < nnz; ++k) {
                co[k] = c.matrix.columns_data()[k];
                va[k] = c.matrix.values_data()[k];
            }
            for (std::size_t i = 0; i < n; ++i) {
                rhs[i] = c.rhs(i);
                guess[i] = c.initial_solution(i);
            }
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/cg_solver.h:591-603 solve_cg without a preconditioner object:
// the solver's own diagonal scaling (the legacy overload).
extern "C" int ref_solve_cg_internal(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                     const double* rhs, double* x, int64_t max_iterations, double tolerance,
                                     ref_report_t* report) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n)), xv(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            b(i) = rhs[i];
            xv(i) = x[i];
        }
        const SolverResult r = solve_cg(A, b, xv, static_cast<std::size_t>(max_iterations), tolerance);
        for (int64_t i = 0; i < n; ++i) x[i] = xv(i);
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->status = static_cast<int32_t>(r.status);
            report->iterations = static_cast<int64_t>(r.iterations);
            report->residual = r.residual;
            report->residual_relative = r.residual_relative;
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/solvers/scalar_diffusion.h:177-210 apply_reference_cell_gauge; the
// output CSR has at most nnz + 1 entries and n + 1 offsets.  Returns its nnz.
extern "C" int64_t ref_apply_reference_cell_gauge(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                                  const double* rhs, int64_t ref, double value, int64_t* ro_out,
                                                  int64_t* co_out, double* va_out, double* rhs_out) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        Vector b(static_cast<std::size_t>(n));
        for (int64_t i = 0; i < n; ++i) b(i) = rhs[i];
        const SparseMatrix G = apply_reference_cell_gauge(A, b, static_cast<std::size_t>(ref), value);
        for (std::size_t i = 0; i <= G.n_rows(); ++i) ro_out[i] = G.row_offsets_data()[i];
        for (std::size_t k = 0; k < G.nnz(); ++k) {
            co_out[k] = G.columns_data()[k];
            va_out[k] = G.values_data()[k];
        }
        for (int64_t i = 0; i < n; ++i) rhs_out[i] = b(i);
        cfdx_ref::g_error.clear();
        return static_cast<int64_t>(G.nnz());
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/solvers/scalar_diffusion.h:294-340 solve_poisson_mixed (the apps/poisson
// driver): types NULL = all Dirichlet, else 0 Dirichlet / 1 Neumann per face.
extern "C" int ref_solve_poisson_mixed(const ref_mesh_t* m, const double* bc, const int32_t* types, double gamma,
                                       const double* source, int64_t max_iterations, double tolerance,
                                       int64_t reference_cell, double reference_value, double* x,
                                       ref_report_t* report) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        PoissonBoundaryCondition boundary = PoissonBoundaryCondition::mixed(mesh.n_faces());
        for (std::size_t f = 0; f < mesh.n_faces(); ++f) {
            boundary.face_values[f] = bc[f];
            boundary.face_types[f] = (types && types[f] == 1) ? PoissonBoundaryType::NEUMANN
                                                               : PoissonBoundaryType::DIRICHLET;
        }
        const std::vector<double> src(source, source + m->n_cells);
        ScalarDiffusionConfig config;
        config.diffusivity = gamma;
        config.max_iterations = static_cast<std::size_t>(max_iterations);
        config.tolerance = tolerance;
        config.gauge.reference_cell = static_cast<std::size_t>(reference_cell);
        config.gauge.reference_value = reference_value;
        const ScalarDiffusionResult r = solve_poisson_mixed(mesh, boundary, src, config);
        for (int64_t i = 0; i < m->n_cells; ++i) x[i] = r.solution(i);
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->status = static_cast<int32_t>(r.linear_result.status);
            report->iterations = static_cast<int64_t>(r.linear_result.iterations);
            report->residual = r.linear_result.residual;
            report->residual_relative = r.linear_result.residual_relative;
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/matrix_diagnostics.h:285  measure_matrix_characteristics
// out_d: equations, average_nnz_per_row, coefficient_range
// out_flags: square, numerically_symmetric, diagonally_dominant, strongly_scaled,
//            large_diagonal_dynamic_range, strongly_directional_coupling,
//            positive_diagonal, saddle_point
extern "C" int ref_measure_characteristics(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                           int32_t saddle_point, double symmetry_tolerance, double* out_d,
                                           int32_t* out_flags) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        const MatrixCharacteristics c = measure_matrix_characteristics(A, saddle_point != 0, symmetry_tolerance);
        out_d[0] = static_cast<double>(c.equations);
        out_d[1] = c.average_nnz_per_row;
        out_d[2] = c.coefficient_range;
        const bool flags[8] = {c.square, c.numerically_symmetric, c.diagonally_dominant, c.strongly_scaled,
                               c.large_diagonal_dynamic_range, c.strongly_directional_coupling,
                               c.positive_diagonal, c.saddle_point};
        for (int k = 0; k < 8; ++k) out_flags[k] = flags[k] ? 1 : 0;
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/linear_solver_models.h:228  select_linear_solver
// flags as above; req: krylov, preconditioner, gmres_restart, null_space, scaling;
// plan: krylov, preconditioner, null_space, automatic_krylov, automatic_preconditioner
extern "C" int ref_select_linear_solver(int32_t problem, int64_t equations, double average_nnz,
                                        double coefficient_range, const int32_t* flags, const int32_t* req,
                                        double braess_sarazin_alpha, int32_t* plan) {
    try {
        MatrixCharacteristics c;
        c.equations = static_cast<std::size_t>(equations);
        c.average_nnz_per_row = average_nnz;
        c.coefficient_range = coefficient_range;
        c.square = flags[0] != 0;
        c.numerically_symmetric = flags[1] != 0;
        c.diagonally_dominant = flags[2] != 0;
        c.strongly_scaled = flags[3] != 0;
        c.large_diagonal_dynamic_range = flags[4] != 0;
        c.strongly_directional_coupling = flags[5] != 0;
        c.positive_diagonal = flags[6] != 0;
        c.saddle_point = flags[7] != 0;
        LinearSolverRequest r;
        r.krylov = static_cast<KrylovModel>(req[0]);
        r.preconditioner = static_cast<PreconditionerModel>(req[1]);
        r.gmres_restart = req[2];
        r.null_space = static_cast<NullSpaceModel>(req[3]);
        r.scaling = static_cast<LinearScalingModel>(req[4]);
        r.braess_sarazin_alpha = braess_sarazin_alpha;
        const LinearSolverPlan p = select_linear_solver(static_cast<LinearProblemKind>(problem), c, r);
        plan[0] = static_cast<int32_t>(p.krylov);
        plan[1] = static_cast<int32_t>(p.preconditioner);
        plan[2] = static_cast<int32_t>(p.null_space);
        plan[3] = p.automatic_krylov ? 1 : 0;
        plan[4] = p.automatic_preconditioner ? 1 : 0;
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/matrix_diagnostics.h:410  scale_matrix (values keep the input pattern
// when no entry merges; nnz_out receives the scaled matrix's entry count)
extern "C" int ref_scale_matrix(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                int32_t scaling, double zero_tolerance, double* row_scale, double* column_scale,
                                double* scaled_values, int64_t* zero_counts, int64_t* nnz_out) {
    try {
        const SparseMatrix A = cfdx_ref::make_csr(n, ro, co, va);
        const MatrixScalingResult r = scale_matrix(A, static_cast<MatrixScaling>(scaling), zero_tolerance);
        for (int64_t i = 0; i < n; ++i) {
            row_scale[i] = r.row_scale[i];
            column_scale[i] = r.column_scale[i];
        }
        *nnz_out = static_cast<int64_t>(r.matrix.nnz());
        for (std::size_t k = 0; k < r.matrix.nnz(); ++k) scaled_values[k] = r.matrix.values_data()[k];
        zero_counts[0] = static_cast<int64_t>(r.zero_rows);
        zero_counts[1] = static_cast<int64_t>(r.zero_columns);
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

// core/linalg/matrix_diagnostics.h:126  diagnose_matrix
// counts: rows, columns, nnz, finite, structurally_consistent, empty_rows, empty_columns,
//         missing_diagonal, near_zero_diagonal, isolated_dofs, duplicate_entries, connected_components
// values: max_abs_value, min_nonzero_abs_value, max_row_sum, min_nonzero_row_sum, max_column_sum,
//         min_nonzero_column_sum, max_abs_diagonal, min_nonzero_abs_diagonal, diagonal_dynamic_range,
//         row_sum_dynamic_range, column_sum_dynamic_range, minimum_gershgorin_margin
extern "C" int ref_diagnose_matrix(int64_t n_rows, int64_t n_cols, const int64_t* ro, const int64_t* co,
                                   const double* va, double tolerance, int32_t topology, int64_t* counts,
                                   double* values) {
    try {
        std::vector<SparseMatrix::Index> off(ro, ro + n_rows + 1), col(co, co + ro[n_rows]);
        std::vector<double> val(va, va + ro[n_rows]);
        const SparseMatrix A = SparseMatrix::from_sorted_csr(static_cast<std::size_t>(n_rows),
                                                             static_cast<std::size_t>(n_cols), std::move(off),
                                                             std::move(col), std::move(val));
        const MatrixDiagnostics d = diagnose_matrix(A, tolerance, topology != 0);
        const int64_t c[12] = {static_cast<int64_t>(d.rows), static_cast<int64_t>(d.columns),
                               static_cast<int64_t>(d.nnz), d.finite ? 1 : 0, d.structurally_consistent ? 1 : 0,
                               static_cast<int64_t>(d.empty_rows), static_cast<int64_t>(d.empty_columns),
                               static_cast<int64_t>(d.missing_diagonal), static_cast<int64_t>(d.near_zero_diagonal),
                               static_cast<int64_t>(d.isolated_dofs), static_cast<int64_t>(d.duplicate_entries),
                               static_cast<int64_t>(d.connected_components)};
        const double v[12] = {d.max_abs_value, d.min_nonzero_abs_value, d.max_row_sum, d.min_nonzero_row_sum,
                              d.max_column_sum, d.min_nonzero_column_sum, d.max_abs_diagonal,
                              d.min_nonzero_abs_diagonal, d.diagonal_dynamic_range, d.row_sum_dynamic_range,
                              d.column_sum_dynamic_range, d.minimum_gershgorin_margin};
        for (int k = 0; k < 12; ++k) {
            counts[k] = c[k];
            values[k] = v[k];
        }
        cfdx_ref::g_error.clear();
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}
