/*
 * cfdxg.h -- C ABI of the B200-native CFDX pressure-correction hot path.
 *
 * One shared library (cfdx_dev_b200/_lib/libcfdxg.so) exports these entry
 * points.  Signatures use plain pointers, sizes and POD structs only.  Every
 * function returns an int status and never throws across the ABI:
 *
 *   >= 0 : mirrors the reference's SolverStatus (core/linalg/solver_status.h:18)
 *          CFDXG_CONVERGED, CFDXG_MAX_ITER_REACHED, CFDXG_DIVERGED,
 *          CFDXG_NOT_APPLICABLE (solves); 0 = success for everything else.
 *   <  0 : CFDXG_ERR_* (bad argument, CUDA failure, failed setup, ...); the
 *          message is available from cfdxg_last_error(ctx).
 *
 * Array arguments are host or device pointers as stated by an explicit
 * `mem` flag (CFDXG_MEM_HOST / CFDXG_MEM_DEVICE).  Vector fields are SoA
 * (x block, then y, then z).  All device work is ordered on the context's
 * CUDA stream; host-memory calls synchronise before returning.
 *
 * The caller owns every array it passes; handles own their device memory.
 * A handle must not be used concurrently from two threads.
 */
#ifndef CFDXG_H
#define CFDXG_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CFDXG_OK 0
#define CFDXG_CONVERGED 0
#define CFDXG_MAX_ITER_REACHED 1
#define CFDXG_DIVERGED 2
#define CFDXG_NOT_APPLICABLE 3
#define CFDXG_ERR_INVALID_ARGUMENT (-1)
#define CFDXG_ERR_CUDA (-2)
#define CFDXG_ERR_SETUP (-3)
#define CFDXG_ERR_NOT_READY (-4)
#define CFDXG_ERR_NONFINITE (-5)
#define CFDXG_ERR_GEOMETRY (-6)
#define CFDXG_ERR_OUT_OF_MEMORY (-7)
#define CFDXG_ERR_IO (-8)

#define CFDXG_MEM_HOST 0
#define CFDXG_MEM_DEVICE 1

/* Krylov / preconditioner / precision choices, numbered as the reference's
 * KrylovModel and PreconditionerModel enums (core/linalg/linear_solver_models.h:20-55). */
#define CFDXG_KRYLOV_AUTO 0         /* KrylovModel::Auto: chosen by select_linear_solver */
#define CFDXG_KRYLOV_CG 1           /* KrylovModel::CG: SPD systems, cg_solver.h */
#define CFDXG_KRYLOV_GMRES 3
#define CFDXG_KRYLOV_FGMRES 4
#define CFDXG_PC_AUTO 0             /* PreconditionerModel::Auto */
#define CFDXG_PC_NONE 1
#define CFDXG_PC_JACOBI 2
#define CFDXG_PC_NATIVE_AMG 6
#define CFDXG_PC_OWN_DIAGONAL 32    /* CG only: the solver's own diagonal scaling, i.e. solve_cg
                                       without a preconditioner object (cg_solver.h:591-603), as
                                       solve_poisson_mixed calls it (scalar_diffusion.h:336-338) */
#define CFDXG_PRECISION_FP64 0      /* the reference's plain FP64 V-cycle */
#define CFDXG_PRECISION_FP32_VCYCLE 1  /* FP32 V-cycle inside FP64 FGMRES */
#define CFDXG_ORTHO_MGS2 0          /* two-pass modified Gram-Schmidt, gmres_solver.h:270-295 */
#define CFDXG_ORTHO_CGS2 1          /* two-pass classical Gram-Schmidt (no reference counterpart) */
/* LinearProblemKind (core/linalg/linear_solver_models.h:11-18) */
#define CFDXG_PROBLEM_GENERAL 0
#define CFDXG_PROBLEM_PRESSURE_POISSON 1
#define CFDXG_PROBLEM_DIFFUSION 2
#define CFDXG_PROBLEM_MOMENTUM 3
#define CFDXG_PROBLEM_SCALAR_TRANSPORT 4
#define CFDXG_PROBLEM_COUPLED_PRESSURE_VELOCITY 5
/* LinearScalingModel (core/linalg/linear_solver_models.h:61) */
#define CFDXG_SCALING_NONE 0
#define CFDXG_SCALING_ROW 1
#define CFDXG_SCALING_COLUMN 2
#define CFDXG_SCALING_ROW_COLUMN 3
#define CFDXG_SCALING_SYMMETRIC_DIAGONAL 4
/* NullSpaceModel (core/linalg/linear_solver_models.h:59) */
#define CFDXG_NULL_SPACE_NONE 0
#define CFDXG_NULL_SPACE_CONSTANT 1

typedef struct cfdxg_context cfdxg_context;
typedef struct cfdxg_mesh cfdxg_mesh;
typedef struct cfdxg_matrix cfdxg_matrix;
typedef struct cfdxg_amg cfdxg_amg;
typedef struct cfdxg_mpnn cfdxg_mpnn;

/* ------------------------------------------------------------------------ */
/* context                                                                  */
/* ------------------------------------------------------------------------ */
/* New: the reference runs on the host thread; the context binds a CUDA
 * device and stream (runtime/gpu/cuda_poisson.cu:143 creates neither). */
int cfdxg_context_create(int32_t device, cfdxg_context** out);
int cfdxg_context_destroy(cfdxg_context* ctx);
/* Message of the last failing call on this context ("" after success).
 * Mirrors NativeAMGPreconditioner::last_error (core/linalg/hypre_amg.h:89-97). */
const char* cfdxg_last_error(const cfdxg_context* ctx);
/* Number of kernels this library launched on the context since creation. */
int64_t cfdxg_kernel_launches(const cfdxg_context* ctx);
int cfdxg_synchronize(cfdxg_context* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order or time
 * their own work around the library's. */
void* cfdxg_context_stream(const cfdxg_context* ctx);

/* Live kernel timing: while enabled, the library brackets its eager launches
 * (fine-level V-cycle kernels, the replay of the coarse-level V-cycle graph,
 * the FP64 operator SpMV, assembly) with CUDA events on its stream and
 * accumulates, per kernel class, launches, device milliseconds and the
 * algorithmic bytes each launch must move (compulsory traffic only).
 * Enabling resets the counters; reading synchronises the stream. */
typedef struct {
    char name[48];
    int64_t launches;
    double total_ms;
    double bytes;
} cfdxg_kernel_profile;
int cfdxg_profile_enable(cfdxg_context* ctx, int32_t on);
int cfdxg_profile_read(cfdxg_context* ctx, cfdxg_kernel_profile* out, int32_t max_entries,
                       int32_t* count);

/* ------------------------------------------------------------------------ */
/* mesh + geometry  (core/mesh/mesh.h:51, core/mesh/ownership.h:25)          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t n_points, n_faces, n_cells;
    const double *px, *py, *pz;      /* n_points */
    const int64_t *face_offsets;     /* n_faces + 1, face -> vertex CSR */
    const int64_t *face_vertices;
    const int64_t *owner;            /* n_faces */
    const int64_t *neighbour;        /* n_faces, -1 on boundary faces */
    const int64_t *cell_offsets;     /* n_cells + 1, cell -> face CSR */
    const int64_t *cell_faces;
    int32_t n_patches;
    const int32_t *patch_of_face;    /* n_faces, -1 on internal faces */
    const int32_t *patch_types;      /* n_patches, reference PatchType values */
} cfdxg_mesh_desc;

/* Copies a host mesh to the device and validates its connectivity. */
int cfdxg_mesh_upload(cfdxg_context* ctx, const cfdxg_mesh_desc* desc, cfdxg_mesh** out);
int cfdxg_mesh_destroy(cfdxg_mesh* mesh);
/* Replaces: build_fv_geometry (physics/finite_volume_transport.h:92-176) and
 * compute_geometry_cache (core/geometry/geometry_cache.h:66-237), which give
 * the same centres, volumes and owner-oriented Sf.  Runs on the GPU. */
int cfdxg_geometry_build(cfdxg_context* ctx, cfdxg_mesh* mesh);
/* Host copies (SoA) of face centres, owner-oriented Sf, cell centres, volumes. */
int cfdxg_geometry_download(cfdxg_context* ctx, const cfdxg_mesh* mesh, double* face_centres,
                            double* face_Sf, double* cell_centres, double* cell_volumes);

/* ------------------------------------------------------------------------ */
/* sparse matrices  (core/linalg/sparse_matrix.h:27)                         */
/* ------------------------------------------------------------------------ */
/* Builds a device CSR from sorted, unique CSR arrays (SparseMatrix::from_sorted_csr,
 * sparse_matrix.h:136-163). */
int cfdxg_matrix_create(cfdxg_context* ctx, int64_t n, const int64_t* row_offsets,
                        const int64_t* columns, const double* values, int32_t mem,
                        cfdxg_matrix** out);
int cfdxg_matrix_destroy(cfdxg_matrix* A);
int cfdxg_matrix_size(const cfdxg_matrix* A, int64_t* n, int64_t* nnz);
int cfdxg_matrix_download(cfdxg_context* ctx, const cfdxg_matrix* A, int64_t* row_offsets,
                          int64_t* columns, double* values);
/* y = A x in FP64, summed per row in CSR order (SparseMatrix::matvec, sparse_matrix.h:180-195). */
int cfdxg_matrix_spmv(cfdxg_context* ctx, const cfdxg_matrix* A, const double* x, double* y,
                      int32_t mem);

/* ------------------------------------------------------------------------ */
/* assembly                                                                  */
/* ------------------------------------------------------------------------ */
/* Replaces assemble_cell_diffusion_matrix (core/solvers/scalar_diffusion.h:39-163):
 * two-point flux Gamma*|Sf|/d, Dirichlet elimination into rhs, Neumann flux,
 * rhs = S*V.  bc_face_values: n_faces, NaN = unprescribed; bc_face_types:
 * n_faces (0 Dirichlet, 1 Neumann) or NULL (all Dirichlet).  Allocates *A_out. */
int cfdxg_assemble_cell_diffusion(cfdxg_context* ctx, cfdxg_mesh* mesh,
                                  const double* bc_face_values, const int32_t* bc_face_types,
                                  double diffusivity, const double* source, int32_t mem,
                                  cfdxg_matrix** A_out, double* rhs);

/* Replaces the pressure-corrector assembly block of solve_steady_incompressible
 * (physics/steady_incompressible_solver.h:8048-8181 with :6485-6500 and the
 * fixed-pressure CSR build :8605-8608): phiHbyA = make_mass_flux(HbyA) (:1842),
 * grad p (:1634), continuity with the Rhie-Chow pressure flux (:1967), face
 * coefficients (:1914), fixed-pressure boundary rows and sources.
 * HbyA, rAU: 3*n_cells SoA; p: n_cells; p_bc_fixed / p_bc_value: per patch.
 * If *A_inout is NULL a matrix is allocated (symbolic pattern built once),
 * otherwise only its values are refreshed.  b: n_cells.  phiHbyA (n_faces)
 * and grad_p (3*n_cells) are optional outputs (NULL to skip). */
int cfdxg_assemble_pressure_correction(cfdxg_context* ctx, cfdxg_mesh* mesh,
                                       const double* HbyA, const double* rAU, const double* p,
                                       double rho, const int32_t* p_bc_fixed,
                                       const double* p_bc_value, int32_t mem,
                                       cfdxg_matrix** A_inout, double* b, double* phiHbyA,
                                       double* grad_p);

/* Replaces make_rhie_chow_mass_flux (physics/steady_incompressible_solver.h:2064-2217),
 * HBYA_PREDICTOR contract, zero-gradient velocity boundaries. flux: n_faces. */
int cfdxg_rhie_chow_flux(cfdxg_context* ctx, cfdxg_mesh* mesh, const double* HbyA,
                         const double* rAU, const double* p, double rho,
                         const int32_t* p_bc_fixed, const double* p_bc_value, int32_t mem,
                         double* flux);

/* No counterpart in the reference.  Same result as cfdxg_rhie_chow_flux, for
 * callers that cannot allocate device memory while they run -- for example a
 * host solver that reserves all GPU memory up front or works under a memory
 * pool that forbids new allocations after start-up (cudaMalloc/cudaFree may
 * also synchronise the device).  This entry point calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch (the cell pressure
 * gradient and the per-patch boundary table) is one static device array of
 * 6 MiB + 512 B that every GPU loading the library holds until exit.
 * Limits: at most 262,144 cells and 32 patches; larger meshes are rejected
 * with CFDXG_ERR_INVALID_ARGUMENT.  HbyA, rAU, p and flux must be device
 * pointers (mesh already uploaded, geometry built); p_bc_fixed / p_bc_value
 * are host arrays of n_patches entries (either may be NULL: no fixed-pressure
 * patch).  Each call makes the context's device current, looks up the
 * array's device address in that context (cudaGetSymbolAddress, which
 * allocates nothing) and gives the caller's current device back before it
 * returns.  The first call on a device can load the library's device code.
 * All calls share the
 * array and it keeps the last call's contents; every call overwrites what it
 * reads, but calls that overlap on the GPU (two streams or threads at once)
 * race on it. */
int cfdxg_rhie_chow_flux_noalloc(cfdxg_context* ctx, cfdxg_mesh* mesh, const double* HbyA,
                                 const double* rAU, const double* p, double rho,
                                 const int32_t* p_bc_fixed, const double* p_bc_value,
                                 double* flux);

/* Replaces the build_hbya step of solve_steady_incompressible
 * (physics/steady_incompressible_solver.h:6430-6465): per velocity component d,
 *   HbyA_d[c] = rAU_d[c] * (rhs_d[c] + gradp_d[c] * V_c - sum_{k: col != c} a_d[k] U_d[col])
 * with the off-diagonal entries of component d's momentum matrix in CSR
 * order.  momentum: three matrices (one per component, may be the same
 * handle) sharing one pattern of n_cells rows; rhs (the momentum equations'
 * right-hand sides), U, gradp, rAU and HbyA: 3*n_cells, component-major.  A
 * non-finite HbyA returns CFDXG_ERR_NONFINITE (the reference throws). */
int cfdxg_build_hbya(cfdxg_context* ctx, cfdxg_mesh* mesh, const cfdxg_matrix* const* momentum,
                     const double* rhs, const double* U, const double* gradp, const double* rAU,
                     int32_t mem, double* HbyA);

/* Replaces gauss_gradient_with_boundary (physics/steady_incompressible_solver.h:1634-1744),
 * default single sweep, distance-weighted interpolation.  grad: 3*n_cells. */
int cfdxg_gauss_gradient(cfdxg_context* ctx, cfdxg_mesh* mesh, const double* p,
                         const int32_t* p_bc_fixed, const double* p_bc_value, int32_t mem,
                         double* grad);

/* ------------------------------------------------------------------------ */
/* Pressure gauge of a pure-Neumann system                                   */
/* ------------------------------------------------------------------------ */
/* CFDXG_GAUGE_ELIMINATE replaces the pure-Neumann branch of the pressure
 * corrector (physics/steady_incompressible_solver.h:8617-8654): the
 * principal submatrix without row and column ref (later indices shift down
 * by one) and the right-hand side without entry ref; cfdxg_gauge_expand then
 * gives the full correction, 0 at ref.  With one unknown the reference keeps
 * the trivial equation p = 0 instead (:8610-8616); create refuses n == 1.
 * CFDXG_GAUGE_IDENTITY_ROW replaces apply_reference_cell_gauge
 * (core/solvers/scalar_diffusion.h:177-210): row and column ref removed, a
 * unit diagonal at (ref, ref), rhs_i -= a_i,ref * value, rhs_ref = value.
 * The plan holds the output pattern (built once, on the host, from the input
 * pattern); cfdxg_gauge_apply gathers values and right-hand side on the
 * device, creating *gauged on its first call and refreshing its values after
 * (a matrix of another pattern is refused).  rhs_out must not alias rhs for
 * the elimination. */
#define CFDXG_GAUGE_ELIMINATE 0
#define CFDXG_GAUGE_IDENTITY_ROW 1
typedef struct cfdxg_gauge cfdxg_gauge;
int cfdxg_gauge_create(cfdxg_context* ctx, const cfdxg_matrix* A, int32_t mode, int64_t ref, double value,
                       cfdxg_gauge** out);
int cfdxg_gauge_apply(cfdxg_context* ctx, const cfdxg_gauge* g, const cfdxg_matrix* A, const double* rhs,
                      int32_t mem, cfdxg_matrix** gauged, double* rhs_out);
int cfdxg_gauge_expand(cfdxg_context* ctx, const cfdxg_gauge* g, const double* x_reduced, int32_t mem, double* x);
int cfdxg_gauge_size(const cfdxg_gauge* g, int64_t* n_out, int64_t* nnz_out);
int cfdxg_gauge_destroy(cfdxg_gauge* g);

/* ------------------------------------------------------------------------ */
/* native AMG preconditioner                                                 */
/* Replaces NativeBoomerAMGPreconditioner (core/linalg/hypre_amg.h:26-101,    */
/* hypre_amg.cpp:163-330): setup / update_values / apply / name / last_error. */
/* ------------------------------------------------------------------------ */
typedef struct {
    double omega;                    /* 0.7 (Balanced policy, hypre_amg.cpp:172) */
    int32_t pre_sweeps;              /* fine-level sweeps; -1 (default): 6 for the FP64 cycle */
    int32_t post_sweeps;             /* (the reference's Balanced policy), 3 for the FP32 cycle */
    double strength_threshold;       /* 0.25 */
    int32_t max_levels;              /* 25 */
    int32_t require_smoother_certificate; /* 1 for CG plans, 0 for GMRES/FGMRES */
    int32_t precision;               /* CFDXG_PRECISION_* of the V-cycle */
    int32_t coarse_dense_limit;      /* FP32 V-cycle: the cycle ends at the first level with
                                        <= this many rows (6000) in a dense inverse, formed
                                        in FP64 (LU with partial pivoting) and stored
                                        FP32; at 64^3 this is the 5,287-row level */
    int32_t reference_order;         /* 1: every row sum in CSR order, so the FP64
                                        V-cycle is bit-identical to the reference's;
                                        0 (default): levels with long rows use a
                                        cooperative, fixed-order (deterministic) row
                                        reduction */
    int32_t coarse_pre_sweeps;       /* pre / post sweeps on levels >= 1; -1 (default):   */
    int32_t coarse_post_sweeps;      /* FP64 cycle -- pre_sweeps / post_sweeps, as in the
                                        reference; FP32 cycle -- 0 / 1 (the fine level keeps
                                        pre_sweeps / post_sweeps).  With 0 pre-sweeps a level
                                        restricts its right-hand side directly (x = 0). */
    int32_t narrow_columns;          /* 1 (default): short-row levels (one thread per row)
                                        whose every |column - row| fits in 16 bits store int16
                                        column offsets (2 bytes less per nonzero read); 0:
                                        int32 columns everywhere.  The arithmetic is the same
                                        either way. */
    int32_t half_values;             /* FP32 V-cycle only.  1 (default): levels whose rows
                                        are shared by several threads (the dense coarse
                                        operators; not the coarsest) store A as FP16 fractions
                                        of each row's largest magnitude, times that magnitude
                                        in FP32: 2 bytes per nonzero instead of 4, sums stay
                                        FP32.  0: FP32 values everywhere. */
    int32_t dense_fp64;              /* FP32 V-cycle only.  0 (default): the dense coarse
                                        inverse is stored FP32; 1: stored FP64 and applied
                                        in FP64 -- with coarse_dense_limit 2000, the FP64
                                        coarsest-level direct solve of the mixed-precision
                                        configuration (1,933 rows at 64^3). */
    int32_t constant_null_space;     /* 0 (default) / 1: the native AMG's constant_null_space
                                        (hypre_amg.h:35): setup and update_values require every
                                        row sum of the operator to vanish (|row sum| <= 256 eps
                                        max(1, largest absolute row sum),
                                        amg_preconditioner.h:1289-1308); the cycle removes the
                                        mean from its input and output, after every sweep,
                                        the restriction and the prolongation, and solves the
                                        <= 16-row coarsest level bordered by a row and a column
                                        of ones (:1191-1203, 2369-2443, 2564-2666).  With
                                        reference_order the means are summed in index order,
                                        so the FP64 cycle is the reference's bit for bit. */
    double coarse_drop_tolerance;    /* FP32 V-cycle only (0 with reference_order).  theta > 0
                                        (default 0.02): the smoothing operator of every level
                                        between the fine and the coarsest keeps its diagonal and
                                        the off-diagonal entries with |a_ij| >= theta * max over
                                        k != i of |a_ik|; each dropped entry is added to its
                                        row's diagonal, so row sums are unchanged.  The Galerkin
                                        hierarchy, its transfers and the FP64 Krylov operator are
                                        untouched: only the FP32 preconditioner changes, and
                                        the solve stops on the same FP64 true residual.  At
                                        64^3 theta = 0.02 keeps 17% of those levels' nonzeros
                                        at the same FGMRES iteration count.  The kept pattern
                                        is fixed at setup; a numeric refresh re-forms its
                                        values and diagonals.  0: the Galerkin operators. */
} cfdxg_amg_options;

int cfdxg_amg_options_default(cfdxg_amg_options* opts);
/* ctx may be NULL (host-only use). */
int cfdxg_amg_create(cfdxg_context* ctx, const cfdxg_amg_options* opts, cfdxg_amg** out);
int cfdxg_amg_destroy(cfdxg_amg* amg);
/* Preconditioner::setup (core/linalg/preconditioner.h:22) */
int cfdxg_amg_setup(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A);
/* Preconditioner::update_values (preconditioner.h:26; hypre_amg.cpp:238-281,
 * amg_preconditioner.h:245-314) -- unchanged pattern only.  The Galerkin
 * products, inverse diagonals and damping are recomputed on the device in the
 * reference's order (bit-identical to the host restatement); on failure
 * (pruned coarse pattern changed, zero diagonal) the hierarchy is unchanged
 * and the status is CFDXG_ERR_SETUP, as the reference's returns false. */
int cfdxg_amg_update_values(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A);
/* Preconditioner::apply (preconditioner.h:27): z = one V-cycle applied to r */
int cfdxg_amg_apply(cfdxg_context* ctx, cfdxg_amg* amg, const double* r, double* z, int32_t mem);
const char* cfdxg_amg_name(const cfdxg_amg* amg);          /* preconditioner.h:28 */
const char* cfdxg_amg_last_error(const cfdxg_amg* amg);    /* hypre_amg.h:97 */
/* Hierarchy diagnostics (hypre_amg.h:66-73 hierarchy_level_sizes/_nnz, smoother omega). */
int32_t cfdxg_amg_num_levels(const cfdxg_amg* amg);
double cfdxg_amg_omega(const cfdxg_amg* amg);
int cfdxg_amg_level_info(const cfdxg_amg* amg, int32_t level, int64_t* n_rows, int64_t* nnz,
                         int64_t* p_nnz);
/* Host copies of one level: A (CSR), inverse diagonal, prolongation (CSR),
 * aggregate (strongest interpolation column per fine row, amg_preconditioner.h:349). */
int cfdxg_amg_export_level(const cfdxg_amg* amg, int32_t level, int64_t* row_offsets,
                           int64_t* columns, double* values, double* inv_diag,
                           int64_t* p_offsets, int64_t* p_columns, double* p_values,
                           int64_t* aggregate);
double cfdxg_amg_setup_seconds(const cfdxg_amg* amg);
/* Host-only hierarchy construction from host CSR arrays, without a device
 * upload (ctx may be NULL): the same setup as cfdxg_amg_setup, for
 * inspection and parity checks on machines without a GPU.  The handle can
 * be exported from but not applied. */
int cfdxg_amg_setup_host(cfdxg_amg* amg, int64_t n, const int64_t* row_offsets,
                         const int64_t* columns, const double* values);
/* Host-only numeric refresh of a cfdxg_amg_setup_host hierarchy
 * (amg_preconditioner.h:245-314 update_values): same pattern, new values. */
int cfdxg_amg_update_values_host(cfdxg_amg* amg, int64_t n, const int64_t* row_offsets,
                                 const int64_t* columns, const double* values);

/* ------------------------------------------------------------------------ */
/* Krylov solves                                                             */
/* ------------------------------------------------------------------------ */
/* Mirrors LinearSolverRequest (core/linalg/linear_solver_models.h:164-189),
 * KrylovControls (core/linalg/krylov_controls.h:10-26) and the precision /
 * learned-preconditioner choices of this library. */
typedef struct {
    int32_t krylov;                  /* CFDXG_KRYLOV_CG / _GMRES / _FGMRES */
    int32_t preconditioner;          /* CFDXG_PC_* */
    int32_t gmres_restart;           /* 40 in the reference's request default */
    int32_t precision;               /* CFDXG_PRECISION_* */
    int32_t restart_min;             /* 10 */
    int32_t restart_max;             /* 512 */
    int32_t adaptive_restart;        /* 1 */
    int32_t residual_replacement;    /* 1 */
    int64_t residual_replacement_period; /* 50 */
    double residual_replacement_gap_ratio; /* 10 */
    double target_reduction_per_cycle;     /* 0.1 */
    cfdxg_mpnn* learned;             /* NULL, or a trained network applied before the V-cycle */
    int32_t learned_applications;    /* the learned stage serves the first this-many Arnoldi
                                        vectors of each restart cycle (the V-cycle alone the
                                        rest); 0: every application.  Default 1. */
    int32_t orthogonalization;       /* CFDXG_ORTHO_MGS2 (default, the reference's order) or
                                        CFDXG_ORTHO_CGS2: h = V^T w, w -= V h, twice -- the same
                                        projections in 4 passes over the basis per Arnoldi step
                                        instead of 4(j+1); rounding differs from MGS2's */
    int32_t problem;                 /* CFDXG_PROBLEM_* (default PRESSURE_POISSON): steers the
                                        automatic choice and the model checks of
                                        select_linear_solver */
    int32_t scaling;                 /* CFDXG_SCALING_* (default NONE): cfdxg_solve_linear_system
                                        solves the scaled system to 0.1 tolerance and certifies
                                        the unscaled one (linear_solver_dispatch.h:302-328,
                                        466-490); CG takes NONE or SYMMETRIC_DIAGONAL only */
    int32_t null_space;              /* CFDXG_NULL_SPACE_* (default NONE).  CONSTANT: the
                                        projected solves of linear_solver_dispatch.h:354-400 for
                                        a singular pure-Neumann pressure / diffusion operator --
                                        GMRES / FGMRES run solve_projected_gmres
                                        (projected_gmres.h:84-150: FGMRES on P A P with the
                                        preconditioner P M P, P v = v - (v.e)e, e the normalised
                                        ones vector), CG the projected CG of cg_solver.h; the
                                        native AMG is built with constant_null_space.  b must
                                        be compatible (|b.e| <= 1e-14 + 1e-12 ||b||) and A e = 0
                                        (and A^T e = 0 for GMRES) to 1e-12 ||A||_F, else
                                        CFDXG_NOT_APPLICABLE with x untouched.  Not combined
                                        with scaling or the learned stage; the unprojected FP64
                                        residual still certifies the result. */
} cfdxg_request;

/* Mirrors SolverResult (core/linalg/solver_status.h:45-72) + LinearSolveReport. */
typedef struct {
    int32_t status;
    int64_t iterations;
    double residual;
    double residual_relative;
    double physical_residual_relative;
    int64_t residual_replacements;
    double max_true_recursive_gap;
    double setup_seconds;
    double solve_seconds;
    int64_t preconditioner_applications;
    int64_t learned_fallbacks;
    int32_t plan_krylov;             /* the Krylov model that ran (KrylovModel numbering) */
    int32_t plan_preconditioner;     /* the preconditioner model that ran */
} cfdxg_report;

int cfdxg_request_default(cfdxg_request* req);

/* Replaces solve_linear_system (core/linalg/linear_solver_dispatch.h:227-492) for
 * scalar pressure systems.  With krylov or
 * preconditioner CFDXG_*_AUTO it first measures the matrix and selects the
 * plan (cfdxg_measure_matrix_characteristics, cfdxg_select_linear_solver, on the
 * host); a plan whose model this library does not provide (BiCGStab, ILU0, ...)
 * returns CFDXG_NOT_APPLICABLE with x untouched and the plan in
 * cfdxg_plan_reason().  Then it builds the requested
 * preconditioner (AMG setup inside, as the reference), solves with
 * right-preconditioned GMRES/FGMRES or with CG (cg_solver.h:45-560), then
 * certifies the FP64 physical residual.  CG first measures the matrix
 * (matrix_diagnostics.h:317-355): not symmetric within 1e-12 max(1, max|a|),
 * or a diagonal that is not positive, returns CFDXG_NOT_APPLICABLE with x
 * untouched (linear_solver_dispatch.h:259-267); its AMG keeps the smoother
 * certificate and is set up only when the initial residual has not already
 * converged.  CG takes no learned stage. */
int cfdxg_solve_linear_system(cfdxg_context* ctx, const cfdxg_matrix* A, const double* rhs,
                              double* x, int32_t mem, const cfdxg_request* req,
                              int64_t max_iterations, double tolerance, cfdxg_report* report);

/* Replaces solve_gmres / solve_fgmres with an already set-up preconditioner
 * (core/linalg/gmres_solver.h:28-600, 690-757, setup_preconditioner = false).
 * amg may be NULL (identity).  With req->krylov == CFDXG_KRYLOV_CG it runs
 * solve_cg(A, b, x, preconditioner) (cg_solver.h:605-618) on that hierarchy,
 * or the identity without one.  With req->null_space == CONSTANT: the
 * projected GMRES of solve_projected_gmres without its setup step, or
 * solve_cg_prepared with the projector (cg_solver.h:653-666). */
int cfdxg_solve_gmres(cfdxg_context* ctx, const cfdxg_matrix* A, cfdxg_amg* amg,
                      const double* rhs, double* x, int32_t mem, const cfdxg_request* req,
                      int64_t max_iterations, double tolerance, cfdxg_report* report);

/* ------------------------------------------------------------------------ */
/* Automatic solver selection (host-only; no device needed)                  */
/* ------------------------------------------------------------------------ */
/* measure_matrix_characteristics (core/linalg/matrix_diagnostics.h:285-358). */
typedef struct {
    int64_t equations;
    double average_nnz_per_row;
    double coefficient_range;        /* max|a| / min nonzero |a| (1 when undefined) */
    int32_t square;
    int32_t numerically_symmetric;   /* |a_ij - a_ji| <= tol * max(1, max|a|) */
    int32_t diagonally_dominant;     /* min Gershgorin margin >= -1e-14 max(1, max|a_ii|) */
    int32_t strongly_scaled;         /* coefficient_range >= 1e8 */
    int32_t large_diagonal_dynamic_range;  /* max|a_ii| / min nonzero |a_ii| >= 1e4 */
    int32_t strongly_directional_coupling; /* a row whose negative couplings differ by >= 1e3 */
    int32_t positive_diagonal;
    int32_t saddle_point;            /* given by the caller */
} cfdxg_matrix_characteristics;
/* The fields of LinearSolverRequest that select_linear_solver reads. */
typedef struct {
    int32_t krylov;                  /* KrylovModel 0..7 (0 = auto) */
    int32_t preconditioner;          /* PreconditionerModel 0..22 (0 = auto) */
    int32_t gmres_restart;
    int32_t null_space;              /* NullSpaceModel: 0 none, 1 constant */
    int32_t scaling;                 /* LinearScalingModel 0..4 */
    double braess_sarazin_alpha;     /* 1 by default */
} cfdxg_plan_request;
/* LinearSolverPlan (linear_solver_models.h:206-214); reason is this
 * library's own wording. */
typedef struct {
    int32_t problem;
    int32_t krylov;
    int32_t preconditioner;
    int32_t null_space;
    int32_t automatic_krylov;
    int32_t automatic_preconditioner;
    char reason[512];
} cfdxg_solver_plan;

/* Characteristics of a square CSR matrix (columns strictly increasing in each
 * row; symmetry_tolerance finite and >= 0, 1e-12 in the dispatcher).  A
 * non-finite value leaves the coefficient evidence at its defaults, as the
 * reference's diagnosis of an inconsistent matrix does. */
int cfdxg_measure_matrix_characteristics(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                                         const double* values, int32_t saddle_point,
                                         double symmetry_tolerance, cfdxg_matrix_characteristics* out);
/* select_linear_solver (core/linalg/linear_solver_models.h:228-425): the same
 * plan for every problem kind, characteristics and request; where the
 * reference throws std::invalid_argument this returns
 * CFDXG_ERR_INVALID_ARGUMENT with the reason in cfdxg_plan_last_error(). */
int cfdxg_select_linear_solver(int32_t problem, const cfdxg_matrix_characteristics* characteristics,
                               const cfdxg_plan_request* request, cfdxg_solver_plan* plan);
const char* cfdxg_plan_last_error(void);
/* scale_matrix (core/linalg/matrix_diagnostics.h:410-490) of a square CSR
 * matrix: scaling CFDXG_SCALING_* (LinearScalingModel numbering); writes the
 * row and column scales (n each), the scaled values (nnz, the input pattern)
 * and, in zero_counts[0..1], the rows and columns left unscaled because their
 * maximum magnitude (or |diagonal|) is <= zero_tolerance. */
int cfdxg_scale_matrix(int64_t n, const int64_t* row_offsets, const int64_t* columns, const double* values,
                       int32_t scaling, double zero_tolerance, double* row_scale, double* column_scale,
                       double* scaled_values, int64_t* zero_counts);
/* diagnose_matrix (core/linalg/matrix_diagnostics.h:126-280) of an n_rows x
 * n_cols CSR matrix: counts and coefficient ranges as the reference's
 * MatrixDiagnostics (:23-59).  A matrix that is not consistent (offsets,
 * columns in range and strictly increasing, finite values) returns with
 * structurally_consistent = finite = 0 and the other fields at their
 * defaults, as the reference does. */
typedef struct {
    int64_t rows, columns, nnz;
    int32_t finite, structurally_consistent;
    int64_t empty_rows, empty_columns, missing_diagonal, near_zero_diagonal, isolated_dofs, duplicate_entries;
    double max_abs_value, min_nonzero_abs_value;
    double max_row_sum, min_nonzero_row_sum, max_column_sum, min_nonzero_column_sum;
    double max_abs_diagonal, min_nonzero_abs_diagonal;
    double diagonal_dynamic_range, row_sum_dynamic_range, column_sum_dynamic_range;
    double minimum_gershgorin_margin;   /* NaN for a rectangular matrix */
    int64_t connected_components;       /* of the bipartite row/column graph; 0 without topology */
} cfdxg_matrix_diagnostics;
int cfdxg_diagnose_matrix(int64_t n_rows, int64_t n_cols, const int64_t* row_offsets, const int64_t* columns,
                          const double* values, double diagonal_relative_tolerance, int32_t include_topology,
                          cfdxg_matrix_diagnostics* out);
/* The plan and its reason of the last cfdxg_solve_linear_system on the context. */
const char* cfdxg_plan_reason(const cfdxg_context* ctx);

/* ------------------------------------------------------------------------ */
/* learned message-passing preconditioner (no reference counterpart)          */
/* ------------------------------------------------------------------------ */
/* A 4-round, 32-feature message-passing network on the mesh's cell-face
 * graph; BF16 weights, FP32 state and accumulation. Applied before the AMG
 * V-cycle inside FGMRES; plain AMG is used whenever it fails to reduce the
 * FP64 true residual. */
int cfdxg_mpnn_create(cfdxg_context* ctx, uint64_t seed, cfdxg_mpnn** out);
int cfdxg_mpnn_destroy(cfdxg_mpnn* net);
int cfdxg_mpnn_num_parameters(const cfdxg_mpnn* net, int64_t* count);
/* Host FP32 copies of the master weights (BF16 copies are derived from them). */
int cfdxg_mpnn_get_parameters(cfdxg_context* ctx, const cfdxg_mpnn* net, float* params);
int cfdxg_mpnn_set_parameters(cfdxg_context* ctx, cfdxg_mpnn* net, const float* params);
int cfdxg_mpnn_save(cfdxg_context* ctx, const cfdxg_mpnn* net, const char* path);
int cfdxg_mpnn_load(cfdxg_context* ctx, cfdxg_mpnn* net, const char* path);
/* Binds the network to a mesh + matrix (graph features: volume, a_P, face area/distance). */
int cfdxg_mpnn_bind(cfdxg_context* ctx, cfdxg_mpnn* net, cfdxg_mesh* mesh, const cfdxg_matrix* A,
                    const double* a_P, int32_t mem);
/* y = N(r) for one residual (FP64 in/out). */
int cfdxg_mpnn_apply(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, double* y, int32_t mem);
/* One Adam step on a batch of (residual, error) pairs: loss = mean over pairs of
 * (e - N(r))^T A (e - N(r)) / (e^T A e).  r, e: batch * n_cells, row-major. */
int cfdxg_mpnn_train_step(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e,
                          int32_t batch, float learning_rate, int32_t mem, double* loss);
/* Sets the V-cycle M the network is trained in front of (NULL: the network
 * alone).  With M the loss of a pair is that of the composed preconditioner
 * z = N(r) + M(r - A N(r)):  ||(I - M A)(e - N(r))||_A^2 / ||(I - M A) e||_A^2,
 * i.e. below 1 exactly when the learned stage improves on the V-cycle alone.
 * M must be symmetric (damped-Jacobi V(k,k) with Galerkin coarse levels is). */
int cfdxg_mpnn_set_vcycle(cfdxg_context* ctx, cfdxg_mpnn* net, cfdxg_amg* amg);
/* Loss and parameter gradient without an update (for gradient checks). */
int cfdxg_mpnn_loss_grad(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e,
                         int32_t batch, int32_t mem, double* loss, float* grad);

/* ------------------------------------------------------------------------ */
/* Linear-system replay files (".cfdxlin")                                   */
/* Replaces write_linear_system_capture / read_linear_system_capture         */
/* (core/linalg/linear_system_capture.h:170-231, :233-284): the same text     */
/* format (FP64 bit patterns in hex, FNV-1a checksum), so a pressure system   */
/* captured by CFDX replays here bit for bit and files written here are      */
/* byte-identical to the reference writer's.  Host-only; no device needed.   */
/* ------------------------------------------------------------------------ */
typedef struct cfdxg_capture cfdxg_capture;
typedef struct {
    int32_t problem;                 /* LinearProblemKind 0..5 (General, PressurePoisson, ...) */
    int32_t null_space;              /* NullSpaceModel: 0 none, 1 constant */
    int32_t scaling;                 /* LinearScalingModel 0..4 */
    int64_t n;                       /* rows (= columns) */
    int64_t nnz;
    int64_t max_iterations;          /* 1 .. 1e8 */
    double tolerance;                /* > 0, finite */
    uint64_t checksum;               /* the file's FNV-1a checksum */
} cfdxg_capture_info;

/* Reads and verifies a capture (format, limits rows <= 2e6 and nnz <= 1e8,
 * CSR invariants, finite values, checksum).  CFDXG_ERR_IO with the reason in
 * cfdxg_capture_last_error() on any failure; *out is then NULL. */
int cfdxg_capture_read(const char* path, cfdxg_capture** out, cfdxg_capture_info* info);
/* Copies the arrays out (sizes n + 1, nnz, nnz, n, n); NULL skips an array. */
int cfdxg_capture_export(const cfdxg_capture* c, int64_t* row_offsets, int64_t* columns, double* values,
                         double* rhs, double* initial_solution);
/* Writes a capture of a host CSR system.  info supplies problem, null_space,
 * scaling, max_iterations and tolerance; n, nnz and checksum are written back.
 * Invalid input (non-finite values, unsorted or out-of-range columns, unknown
 * metadata, limits) is refused with CFDXG_ERR_INVALID_ARGUMENT before any
 * file is created; the file appears by rename of "<path>.tmp" once complete. */
int cfdxg_capture_write(const char* path, int64_t n, const int64_t* row_offsets, const int64_t* columns,
                        const double* values, const double* rhs, const double* initial_solution,
                        cfdxg_capture_info* info);
int cfdxg_capture_destroy(cfdxg_capture* c);
/* Reason of the calling thread's last failed capture call. */
const char* cfdxg_capture_last_error(void);

/* ------------------------------------------------------------------------ */
/* Domain decomposition plan (row blocks with halos)                         */
/* New: the reference solves one system on one rank (its MPI layer does not  */
/* reach this path; linear_solver_dispatch.h:227-234 takes the whole        */
/* SparseMatrix).  A plan splits the rows of a square CSR system into       */
/* contiguous blocks ("parts", one or more per GPU) and lists, per part:   */
/*  - its local system: the owned rows with their columns renumbered into   */
/*    the local vector [ghosts below | owned | ghosts above], increasing in  */
/*    the global column order, so every local row keeps the global row's    */
/*    entry order (a local product sums exactly as the global one does);    */
/*  - its diagonal block (owned columns only, owned numbering) for a        */
/*    subdomain preconditioner;                                            */
/*  - per neighbouring part the ghosts it receives (a contiguous slice of    */
/*    the local vector) and the owned rows it sends.                         */
/* Each entry carries the index of the global CSR entry it copies, so a      */
/* numeric refresh is a gather.  Host-only; no device needed.               */
/* ------------------------------------------------------------------------ */
typedef struct cfdxg_domain_plan cfdxg_domain_plan;
typedef struct {
    int64_t row_begin, row_end;      /* owned global rows [row_begin, row_end) */
    int64_t n_local;                 /* local vector length: ghosts + owned columns */
    int64_t owned_offset;            /* local position of col_begin (= ghosts below) */
    int64_t nnz_local;               /* entries of the owned rows */
    int64_t nnz_block;               /* entries in owned columns */
    int32_t n_neighbours;
    int64_t n_recv, n_send;          /* ghost values received / owned values sent */
    int64_t col_begin, col_end;      /* owned columns (= the rows for a square plan) */
    int64_t n_local_rows;            /* rows of the local system: n_local for a square
                                        plan (ghost rows empty), owned rows otherwise */
    int64_t first_row;               /* local row of row_begin: owned_offset or 0 */
} cfdxg_domain_part_info;
typedef struct {                     /* output arrays; NULL skips one */
    int64_t* local_row_offsets;      /* n_local_rows + 1 */
    int64_t* local_columns;          /* nnz_local, local numbering */
    int64_t* local_source;           /* nnz_local, global CSR entry index */
    int64_t* block_row_offsets;      /* (row_end - row_begin) + 1 */
    int64_t* block_columns;          /* nnz_block, column - col_begin */
    int64_t* block_source;           /* nnz_block */
    int32_t* neighbours;             /* n_neighbours, increasing part ids */
    int64_t* recv_offsets;           /* n_neighbours + 1 into ghost_rows */
    int64_t* recv_start;             /* n_neighbours: local position of each slice */
    int64_t* ghost_rows;             /* n_recv global columns, increasing */
    int64_t* send_offsets;           /* n_neighbours + 1 into send_rows */
    int64_t* send_rows;              /* n_send owned column indices (0-based in the part) */
} cfdxg_domain_part_arrays;

/* Builds the plan of an n x n CSR pattern (row offsets, columns strictly
 * increasing in each row) split into `parts` row blocks.  row_splits
 * (parts + 1 increasing offsets from 0 to n) fixes the blocks; NULL splits
 * the rows into blocks of nearly equal entry counts.  Every block must own
 * at least one row.  CFDXG_ERR_INVALID_ARGUMENT with the reason in
 * cfdxg_domain_last_error() on bad input. */
int cfdxg_domain_plan_create(int64_t n, const int64_t* row_offsets, const int64_t* columns, int32_t parts,
                             const int64_t* row_splits, cfdxg_domain_plan** out);
/* The plan of an n_rows x n_cols operator (an AMG transfer: P or P^T) whose
 * rows are split by row_splits and whose input vector by col_splits (both
 * parts + 1 offsets, required): part p owns rows and input entries of its
 * blocks; the local input vector is [ghosts below | owned | ghosts above]. */
int cfdxg_domain_plan_create_rect(int64_t n_rows, int64_t n_cols, const int64_t* row_offsets,
                                  const int64_t* columns, int32_t parts, const int64_t* row_splits,
                                  const int64_t* col_splits, cfdxg_domain_plan** out);
/* Row and column splits (parts + 1 each, NULL skips); returns the number of parts. */
int cfdxg_domain_plan_parts(const cfdxg_domain_plan* plan, int64_t* row_splits, int64_t* col_splits);
int cfdxg_domain_plan_info(const cfdxg_domain_plan* plan, int32_t part, cfdxg_domain_part_info* info);
int cfdxg_domain_plan_export(const cfdxg_domain_plan* plan, int32_t part, const cfdxg_domain_part_arrays* out);
int cfdxg_domain_plan_destroy(cfdxg_domain_plan* plan);
const char* cfdxg_domain_last_error(void);

/* ------------------------------------------------------------------------ */
/* synthetic cases (seeded generators for the benchmark configurations)      */
/* ------------------------------------------------------------------------ */
typedef struct cfdxg_case cfdxg_case;
/* Hex lattice nx*ny*nz on the unit cube, face numbering of the reference's
 * hex fixture (tests/validation/thermal_3d_mesh_v36.h:18-80), patches
 * west,east,south,north,bottom,top = 0..5. */
int cfdxg_case_hex(int64_t nx, int64_t ny, int64_t nz, cfdxg_case** out);
/* Kuhn 6-tet split of an n^3 lattice on the unit cube, face numbering of the
 * reference's tet fixture (tests/validation/radiation_tetrahedral_mesh_v52.h:14-92);
 * interior vertices jittered by U[-jitter*h, jitter*h] per coordinate.
 * Patches xmin,xmax,ymin,ymax,zmin,zmax = 0..5. */
int cfdxg_case_tet(int64_t n, double jitter, uint64_t seed, cfdxg_case** out);
/* Boundary-layer hex nx*ny*nz on [0,lx]x[0,1]x[0,lz]: y spacing dy0*growth^j
 * capped so the column fills [0,1]; x/z interior lines jittered by +-jitter*h. */
int cfdxg_case_boundary_layer(int64_t nx, int64_t ny, int64_t nz, double lx, double lz,
                              double dy0, double growth, double jitter, uint64_t seed,
                              cfdxg_case** out);
int cfdxg_case_destroy(cfdxg_case* c);
/* sizes: n_points, n_faces, n_face_vertices, n_cells, n_cell_faces, n_patches */
int cfdxg_case_sizes(const cfdxg_case* c, int64_t* sizes);
int cfdxg_case_export(const cfdxg_case* c, double* px, double* py, double* pz,
                      int64_t* face_offsets, int64_t* face_vertices, int64_t* owner,
                      int64_t* neighbour, int64_t* cell_offsets, int64_t* cell_faces,
                      int32_t* patch_of_face, int32_t* patch_types);
/* Seeded fields at the given cell centres (SoA 3*n): divergence-free sum of
 * n_modes Fourier modes with amplitude 1/|k|^2 plus U[-perturbation, perturbation]. */
int cfdxg_field_fourier(int64_t n, const double* centres, int32_t n_modes, double perturbation,
                        uint64_t seed, double* u);
/* Seeded per-cell values: log-uniform on [lo, hi] (kind 0) or uniform (kind 1). */
int cfdxg_field_random(int64_t n, int32_t kind, double lo, double hi, uint64_t seed, double* v);

#ifdef __cplusplus
}
#endif
#endif /* CFDXG_H */
