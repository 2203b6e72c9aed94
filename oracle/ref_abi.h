/*
 * ref_abi.h -- C interface of the reference-built oracle (oracle/_ref/libcfdx_ref.so).
 *
 * TEST INFRASTRUCTURE ONLY.  The library behind this header is compiled from
 * the reference's own C++ sources (stevendaix/cfdx_dev, src/cfdx/...) by
 * oracle/Makefile, with the thin adapters in oracle/ref_linalg.cpp and
 * oracle/ref_simple.cpp.  It is the checker for parity tests and the CPU
 * baseline of bench.py; the product never links or calls it.
 *
 * All arrays are flat host arrays.  Vector fields are SoA: x[0..n), y[n..2n),
 * z[2n..3n).  Meshes use int64 indices; neighbour < 0 marks a boundary face.
 */
#ifndef CFDX_REF_ABI_H
#define CFDX_REF_ABI_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n_points, n_faces, n_cells;
    const double *px, *py, *pz;
    const int64_t *face_offsets;   /* n_faces + 1 */
    const int64_t *face_vertices;
    const int64_t *owner;          /* n_faces */
    const int64_t *neighbour;      /* n_faces, -1 on boundary faces */
    const int64_t *cell_offsets;   /* n_cells + 1 */
    const int64_t *cell_faces;
    int32_t n_patches;
    const int32_t *patch_of_face;  /* n_faces, -1 on internal faces */
    const int32_t *patch_types;    /* n_patches, reference PatchType values */
} ref_mesh_t;

typedef struct {
    int32_t status;                /* SolverStatus */
    int64_t iterations;
    double residual;
    double residual_relative;
    double physical_residual_relative;
    double setup_seconds;
    double solve_seconds;
} ref_report_t;

/* last error message of the calling thread (empty when the last call succeeded) */
const char* ref_last_error(void);

/* --- reference mesh fixtures (connectivity pins) --- */
/* tests/validation/radiation_tetrahedral_mesh_v52.h  tetrahedral_mesh(n) */
int ref_fixture_tet_v52_sizes(int64_t n, int64_t* sizes /* points, faces, face_verts, cells, cell_faces */);
int ref_fixture_tet_v52(int64_t n, double* px, double* py, double* pz,
                        int64_t* face_offsets, int64_t* face_vertices,
                        int64_t* owner, int64_t* neighbour,
                        int64_t* cell_offsets, int64_t* cell_faces);

/* --- geometry --- */
/* core/geometry/geometry_cache.h:66  compute_geometry_cache (config-1 path) */
int ref_geometry_cache(const ref_mesh_t* m, double* face_centres, double* face_Sf,
                       double* cell_centres, double* cell_volumes);
/* physics/finite_volume_transport.h:92  build_fv_geometry (SIMPLE path) */
int ref_fv_geometry(const ref_mesh_t* m, double* face_centres, double* face_Sf,
                    double* cell_centres, double* cell_volumes);

/* --- assembly --- */
/* core/solvers/scalar_diffusion.h:39  assemble_cell_diffusion_matrix; returns nnz or -1 */
int64_t ref_assemble_diffusion(const ref_mesh_t* m, const double* bc_face_values,
                               double diffusivity, const double* source,
                               int64_t* row_offsets, int64_t* columns, double* values,
                               double* rhs, double* seconds);

/* physics/steady_incompressible_solver.h:8048-8181 pressure-corrector assembly;
 * p_bc_fixed / p_bc_value are per patch.  returns nnz or -1 */
int64_t ref_simple_assemble(const ref_mesh_t* m, const double* HbyA, const double* rAU,
                            const double* p, double rho,
                            const int32_t* p_bc_fixed, const double* p_bc_value,
                            double* phiHbyA, double* grad_p,
                            int64_t* row_offsets, int64_t* columns, double* values,
                            double* b, double* seconds);

/* physics/steady_incompressible_solver.h:2064  make_rhie_chow_mass_flux */
int ref_rhie_chow_flux(const ref_mesh_t* m, const double* HbyA, const double* rAU,
                       const double* p, double rho,
                       const int32_t* p_bc_fixed, const double* p_bc_value,
                       double* flux);
/* physics/steady_incompressible_solver.h:1634  gauss_gradient_with_boundary */
int ref_gauss_gradient(const ref_mesh_t* m, const double* p,
                       const int32_t* p_bc_fixed, const double* p_bc_value,
                       double* grad);

/* --- native AMG (core/linalg/hypre_amg.cpp:163 setup, Balanced policy) --- */
void* ref_amg_create(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                     const double* values, int32_t require_smoother_certificate,
                     double* seconds);
/* Reference preconditioner around a supplied hierarchy (no setup run); for
 * timing the reference's own V-cycle / GMRES where its setup is infeasible. */
void* ref_amg_create_from_levels(int32_t n_levels, const int64_t* n_rows,
                                 const int64_t* const* row_offsets, const int64_t* const* columns,
                                 const double* const* values, const double* const* inv_diag,
                                 const int64_t* const* p_offsets, const int64_t* const* p_columns,
                                 const double* const* p_values, double omega);
void ref_amg_destroy(void* h);
/* core/linalg/amg_preconditioner.h:245  update_values (same pattern, new values); 1 = refused */
int ref_amg_update_values(void* h, int64_t n, const int64_t* row_offsets, const int64_t* columns,
                          const double* values);
int32_t ref_amg_num_levels(void* h);
double ref_amg_omega(void* h);
int ref_amg_level_sizes(void* h, int32_t level, int64_t* n_rows, int64_t* nnz, int64_t* p_nnz);
int ref_amg_level_matrix(void* h, int32_t level, int64_t* row_offsets, int64_t* columns,
                         double* values, double* inv_diag);
int ref_amg_level_prolongation(void* h, int32_t level, int64_t* row_offsets,
                               int64_t* columns, double* values, int64_t* aggregate);
/* core/linalg/amg_preconditioner.h:1191  apply (one V-cycle, z = M^-1 r) */
int ref_amg_apply(void* h, const double* r, double* z);

/* --- solves --- */
/* core/linalg/linear_solver_dispatch.h:227  solve_linear_system (setup + solve) */
int ref_solve_linear_system(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                            const double* values, const double* rhs, double* x,
                            int32_t krylov, int32_t preconditioner, int32_t restart,
                            int64_t max_iterations, double tolerance, ref_report_t* report);
/* core/linalg/gmres_solver.h:690  solve_gmres with an already set-up AMG */
int ref_solve_gmres_prepared(void* amg, int64_t n, const int64_t* row_offsets,
                             const int64_t* columns, const double* values,
                             const double* rhs, double* x, int32_t restart,
                             int64_t max_iterations, double tolerance,
                             ref_report_t* report);
/* core/linalg/linear_system_capture.h:170 / :233 -- the .cfdxlin replay format */
int ref_write_capture(const char* path, int64_t n, const int64_t* row_offsets, const int64_t* columns,
                      const double* values, const double* rhs, const double* guess, int32_t problem,
                      int32_t null_space, int32_t scaling, int64_t max_iterations, double tolerance);
int ref_read_capture(const char* path, int64_t* meta /* n, nnz, problem, null_space, scaling, max_it */,
                     double* tolerance, int64_t* row_offsets, int64_t* columns, double* values,
                     double* rhs, double* guess);
/* core/linalg/cg_solver.h:591 solve_cg(A, b, x, max_iter, tolerance): CG with its own diagonal */
int ref_solve_cg_internal(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                          const double* rhs, double* x, int64_t max_iterations, double tolerance,
                          ref_report_t* report);
/* core/solvers/scalar_diffusion.h:177-210 apply_reference_cell_gauge (returns the output nnz) */
int64_t ref_apply_reference_cell_gauge(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                                       const double* values, const double* rhs, int64_t ref, double value,
                                       int64_t* ro_out, int64_t* co_out, double* va_out, double* rhs_out);
/* core/solvers/scalar_diffusion.h:294-340 solve_poisson_mixed; types NULL = all Dirichlet */
int ref_solve_poisson_mixed(const ref_mesh_t* m, const double* bc, const int32_t* types, double gamma,
                            const double* source, int64_t max_iterations, double tolerance, int64_t reference_cell,
                            double reference_value, double* x, ref_report_t* report);

/* --- automatic solver selection --- */
/* core/linalg/matrix_diagnostics.h:285  measure_matrix_characteristics
 * out_d: equations, average_nnz_per_row, coefficient_range; out_flags: square,
 * numerically_symmetric, diagonally_dominant, strongly_scaled,
 * large_diagonal_dynamic_range, strongly_directional_coupling, positive_diagonal,
 * saddle_point */
int ref_measure_characteristics(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                                const double* values, int32_t saddle_point, double symmetry_tolerance,
                                double* out_d, int32_t* out_flags);
/* core/linalg/linear_solver_models.h:228  select_linear_solver; -1 where it throws.
 * req: krylov, preconditioner, gmres_restart, null_space, scaling (reference enums);
 * plan: krylov, preconditioner, null_space, automatic_krylov, automatic_preconditioner */
int ref_select_linear_solver(int32_t problem, int64_t equations, double average_nnz,
                             double coefficient_range, const int32_t* flags, const int32_t* req,
                             double braess_sarazin_alpha, int32_t* plan);
/* core/linalg/matrix_diagnostics.h:126  diagnose_matrix (field order in ref_linalg.cpp) */
int ref_diagnose_matrix(int64_t n_rows, int64_t n_cols, const int64_t* row_offsets, const int64_t* columns,
                        const double* values, double tolerance, int32_t topology, int64_t* counts, double* values_out);
/* core/linalg/matrix_diagnostics.h:410  scale_matrix (MatrixScaling numbering) */
int ref_scale_matrix(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                     int32_t scaling, double zero_tolerance, double* row_scale, double* column_scale,
                     double* scaled_values, int64_t* zero_counts, int64_t* nnz_out);
/* one SpMV with SparseMatrix::matvec (sparse_matrix.h:180) */
int ref_spmv(int64_t n, const int64_t* row_offsets, const int64_t* columns,
             const double* values, const double* x, double* y);

#ifdef __cplusplus
}
#endif
#endif
