/*
 * cfdx_oracle.h -- plain-C restatement of the CFDX pressure-correction hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the parity tests, of
 * __graft_entry__.smoke() and of bench.py's CPU legs.  The product never links
 * or calls it.  Every function restates one reference function of
 * stevendaix/cfdx_dev (file:line cited at each declaration) with the same
 * floating-point operation order, so its results are bit-identical to the
 * reference's; tests/test_oracle_pin.py checks that against the reference
 * compiled into oracle/_ref and against the committed fixtures under
 * tests/golden/.  Compiled with -ffp-contract=off (no fused multiply-add).
 *
 * Arrays are flat host arrays; vector fields are SoA (x[0..n), y[n..2n),
 * z[2n..3n)); meshes use int64 indices, neighbour < 0 on boundary faces.
 * Functions return 0 on success and a negative code on invalid input
 * (co_last_error() holds the reason).
 */
#ifndef CFDX_ORACLE_H
#define CFDX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* the reference's PatchType values used by the face loops */
#define CO_PATCH_SYMMETRY 3
#define CO_PATCH_EMPTY 6

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
    const int32_t *patch_types;    /* n_patches */
} co_mesh_t;

typedef struct {
    int32_t status;                /* 0 converged, 1 max iterations, 2 diverged, 3 not applicable */
    int64_t iterations;
    double residual;
    double residual_relative;
    int64_t residual_replacements;
    int64_t preconditioner_applications;
} co_report_t;

const char* co_last_error(void);

/* physics/finite_volume_transport.h:92-176 build_fv_geometry (face fan
 * core/geometry/face_geometry.h:50-90, oriented cell geometry
 * core/geometry/cell_geometry.h:49-147, ensure_face_orientation
 * face_geometry.h:115-127, second cell pass). */
int co_fv_geometry(const co_mesh_t* m, double* face_centres, double* face_Sf,
                   double* cell_centres, double* cell_volumes);

/* physics/steady_incompressible_solver.h:1634-1744 gauss_gradient_with_boundary
 * (single sweep, distance weights, fixed-value / zero-gradient patches). */
int co_gauss_gradient(const co_mesh_t* m, const double* p, const int32_t* fixed,
                      const double* value, double* grad);

/* The corrector block physics/steady_incompressible_solver.h:8048-8181 with
 * make_mass_flux :1842-1905, rhie_chow_pressure_flux_internal :1967-2024,
 * the orthogonal / non-orthogonal face terms :1914-1965 and the directional
 * coefficient :6485-6500; full system with a fixed-pressure patch :8605-8608.
 * CSR: columns sorted per row, diagonal included.  Returns nnz or < 0. */
int64_t co_pressure_assemble(const co_mesh_t* m, const double* HbyA, const double* rAU,
                             const double* p, double rho, const int32_t* fixed,
                             const double* value, double* phiHbyA, double* grad_p,
                             int64_t* row_offsets, int64_t* columns, double* values,
                             double* b);

/* physics/steady_incompressible_solver.h:2064-2217 make_rhie_chow_mass_flux
 * (HBYA_PREDICTOR contract, zero-gradient velocity patches). */
int co_rhie_chow_flux(const co_mesh_t* m, const double* HbyA, const double* rAU,
                      const double* p, double rho, const int32_t* fixed,
                      const double* value, double* flux);

/* core/solvers/scalar_diffusion.h:39-163 assemble_cell_diffusion_matrix;
 * bc_face_values NaN = unprescribed face, bc_types NULL = all Dirichlet
 * (0 Dirichlet, 1 prescribed flux).  Returns nnz or < 0. */
/* The build_hbya step of solve_steady_incompressible
 * (physics/steady_incompressible_solver.h:6430-6465), per velocity component d
 * (SoA arrays of 3*n, d-th block):
 *   HbyA_d[c] = rAU_d[c] * (rhs_d[c] + gradp_d[c] * V_c - sum_{k: col != c} a_d[k] * U_d[col])
 * with the off-diagonal entries of the component's momentum matrix in CSR
 * order.  values: 3 arrays of nnz (one matrix per component, same pattern).
 * Returns -1 on a non-finite HbyA (the reference throws). */
int co_build_hbya(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                  const double* rhs, const double* U, const double* gradp, const double* volumes,
                  const double* rAU, double* HbyA);

int64_t co_assemble_diffusion(const co_mesh_t* m, const double* bc_face_values,
                              const int32_t* bc_types, double diffusivity,
                              const double* source, int64_t* row_offsets,
                              int64_t* columns, double* values, double* rhs);

/* core/linalg/sparse_matrix.h SparseMatrix::matvec: y_i = sum_k a_ik x_k in row order */
void co_spmv(int64_t n, const int64_t* row_offsets, const int64_t* columns,
             const double* values, const double* x, double* y);

/* One AMG V-cycle on a given hierarchy, z = M^-1 r from z = 0:
 * core/linalg/amg_preconditioner.h:1191-1203 apply, :2411-2443 vcycle,
 * :2369-2409 damped-Jacobi smooth, :2564-2666 smooth_coarsest (dense pivoted
 * LU when the last level has <= 16 rows, else 24 sweeps from zero).
 * Level l: n_rows[l], CSR (row_offsets/columns/values)[l], inv_diag[l]; the
 * prolongation of level l (l < n_levels - 1) maps level l+1 to level l. */
typedef struct {
    int32_t n_levels;
    const int64_t* n_rows;
    const int64_t* const* row_offsets;
    const int64_t* const* columns;
    const double* const* values;
    const double* const* inv_diag;
    const int64_t* const* p_offsets;
    const int64_t* const* p_columns;
    const double* const* p_values;
    double omega;
    int32_t pre_sweeps, post_sweeps;
    /* the constant_null_space flag of the native AMG (hypre_amg.h:35,
     * amg_preconditioner.h:1197-1201, 2382, 2406, 2430, 2440, 2590-2664):
     * mean subtraction on the cycle's input and output, after every smoother
     * sweep, after the restriction and after the prolongation; the <= 16-row
     * coarsest level solves the system bordered by a row and column of ones */
    int32_t constant_null_space;
} co_hierarchy_t;

int co_vcycle(const co_hierarchy_t* h, const double* r, double* z);

/* core/linalg/gmres_solver.h:28-600 solve_gmres, right-preconditioned by
 * co_vcycle (h may be NULL: unpreconditioned), KrylovControls defaults of
 * core/linalg/krylov_controls.h:10-26 (adaptive restart [10, 512], residual
 * replacement every 50 iterations with gap ratio 10, target reduction 0.1).
 * x holds the initial guess and receives the solution. */
int co_solve_gmres(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                   const double* values, const co_hierarchy_t* h, const double* b,
                   double* x, int32_t restart, int64_t max_iterations, double tolerance,
                   co_report_t* report);

/* core/linalg/cg_solver.h:45-560 solve_cg_impl, FP64 without a null space:
 * the true residual certifies every iteration, residual replacement as the
 * reference (adaptive with a preconditioner object, the recursive-norm rule
 * without).  preconditioner: CO_CG_INTERNAL_JACOBI -- no object, the solver's
 * own diagonal (the legacy solve_cg overload); CO_CG_IDENTITY, CO_CG_JACOBI,
 * CO_CG_AMG -- the objects solve_linear_system builds for None / Jacobi /
 * NativeAMG (linear_solver_dispatch.h:169-189), AMG applying co_vcycle on h.
 * x holds the initial guess and receives the solution. */
#define CO_CG_INTERNAL_JACOBI 0
#define CO_CG_IDENTITY 1
#define CO_CG_JACOBI 2
#define CO_CG_AMG 6
int co_solve_cg(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                const double* values, int32_t preconditioner, const co_hierarchy_t* h,
                const double* b, double* x, int64_t max_iterations, double tolerance,
                co_report_t* report);

/* The constant null space (core/linalg/null_space.h, projected_gmres.h).
 * co_null_space_entry: every entry of NullSpaceProjector::constant(n)'s basis
 * vector (null_space.h:58-62: ones over their hypot-accumulated norm).
 * co_null_space_checks: out[0] is_compatible(b) (null_space.h:97-105),
 * out[1] is_null_space(A) (:107-134), out[2] is_bilateral_null_space(A)
 * (projected_gmres.h:53-82), each 0 or 1.
 * co_solve_projected_gmres: solve_projected_gmres (projected_gmres.h:84-150),
 * the right-preconditioned FGMRES of co_solve_gmres on P A P with the
 * preconditioner P M P (h may be NULL: the identity); x untouched and status 3
 * when the checks fail.
 * co_solve_cg_ns: co_solve_cg with the NullSpaceProjector of
 * cg_solver.h:74-79, 93, 149, 203, 262, 295-298, 376, 419, 517, 558
 * (null_space 0: exactly co_solve_cg). */
double co_null_space_entry(int64_t n);
int co_null_space_checks(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                         const double* b, int32_t* out);
int co_solve_projected_gmres(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                             const double* values, const co_hierarchy_t* h, const double* b, double* x,
                             int32_t restart, int64_t max_iterations, double tolerance, co_report_t* report);
int co_solve_cg_ns(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                   int32_t preconditioner, const co_hierarchy_t* h, const double* b, double* x,
                   int64_t max_iterations, double tolerance, int32_t null_space, co_report_t* report);

/* Pressure gauge of a pure-Neumann system.  co_gauge_eliminate: the
 * pure-Neumann branch of the corrector (physics/steady_incompressible_solver.h
 * :8617-8654), the principal submatrix without row/column ref and b without
 * entry ref (returns nnz, outputs sized n, nnz_in, nnz_in, n - 1);
 * co_gauge_expand: the full correction with 0 at ref (:8645-8653);
 * co_gauge_identity_row: core/solvers/scalar_diffusion.h:177-210
 * apply_reference_cell_gauge (returns nnz; outputs sized n + 1, nnz_in + 1,
 * nnz_in + 1, n). */
int64_t co_gauge_eliminate(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                           const double* b, int64_t ref, int64_t* ro_out, int64_t* co_out, double* va_out,
                           double* b_out);
void co_gauge_expand(int64_t n, const double* x_reduced, int64_t ref, double* x);
int64_t co_gauge_identity_row(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                              const double* b, int64_t ref, double value, int64_t* ro_out, int64_t* co_out,
                              double* va_out, double* b_out);

#ifdef __cplusplus
}
#endif
#endif
