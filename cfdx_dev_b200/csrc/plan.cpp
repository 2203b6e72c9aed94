// plan.cpp -- automatic solver selection (host only).
//
// select_solver restates select_linear_solver
// (core/linalg/linear_solver_models.h:228-425): the rule that maps a problem
// kind, the measured matrix characteristics and a request to a Krylov method,
// a preconditioner and a null-space treatment, with the same rejections.  The
// model numbers are the reference's enums (KrylovModel :20-29,
// PreconditionerModel :31-55); availability follows its catalogs (:80-126).
// The reason text is this library's own.
#include "plan.h"

#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

namespace cfdxg {

namespace {

enum Krylov { kAuto = 0, kCG = 1, kBiCGStab = 2, kGMRES = 3, kFGMRES = 4, kKrylovCount = 8 };
enum Pc {
    pAuto = 0, pNone = 1, pJacobi = 2, pILU0 = 4, pNativeAMG = 6, pSmoothedAggregationAMG = 7,
    pAnisotropicLineAMG = 8, pNativeFieldSplit = 11, pCoupledBlockSchur = 12, pPCD = 13, pMGR = 15,
    pAnisotropicLine = 16, pAnisotropicBoomerAMG = 17, pAnisotropicSmoothedAggregationAMG = 18,
    pDirectionalSemiCoarseningAMG = 19, pEnergyMinimizingAMG = 20, pVankaPressurePatch = 21,
    pBraessSarazin = 22, kPcCount = 23
};
enum Problem { General = 0, PressurePoisson = 1, Diffusion = 2, Momentum = 3, ScalarTransport = 4, Coupled = 5 };

const char* const kKrylovNames[kKrylovCount] = {"auto", "cg", "bicgstab", "gmres", "fgmres", "lgmres", "pipecg",
                                                 "pipefgmres"};
const bool kKrylovAvailable[kKrylovCount] = {true, true, true, true, true, false, false, false};
const char* const kPcNames[kPcCount] = {
    "auto", "none", "jacobi", "gauss_seidel", "ilu0", "ilut", "native_amg", "smoothed_aggregation_amg",
    "anisotropic_line_amg", "fsai", "ras", "native_fieldsplit", "coupled_block_schur", "pcd", "lsc", "mgr",
    "anisotropic_line", "anisotropic_boomer_amg", "anisotropic_smoothed_aggregation_amg",
    "directional_semi_coarsening_amg", "energy_minimizing_amg", "vanka_pressure_patch", "braess_sarazin"};
// ilut, fsai, ras and lsc are planned, not available
const bool kPcAvailable[kPcCount] = {true, true, true, true, true, false, true, true, true, false, false, true,
                                     true, true, false, true, true, true, true, true, true, true, true};

bool fail(std::string& why, const std::string& text) {
    why = text;
    return false;
}

}  // namespace

const char* krylov_model_name(int32_t m) { return m >= 0 && m < kKrylovCount ? kKrylovNames[m] : "unknown"; }
const char* preconditioner_model_name(int32_t m) { return m >= 0 && m < kPcCount ? kPcNames[m] : "unknown"; }

bool select_solver(int32_t problem, const cfdxg_matrix_characteristics& c, const cfdxg_plan_request& r,
                   cfdxg_solver_plan& plan, std::string& why) {
    if (problem < General || problem > Coupled) return fail(why, "unknown problem kind");
    if (r.null_space < 0 || r.null_space > 1) return fail(why, "unknown null-space model");
    if (r.scaling < 0 || r.scaling > 4) return fail(why, "unknown scaling model");
    if (r.krylov < 0 || r.krylov >= kKrylovCount) return fail(why, "unknown Krylov model");
    if (r.preconditioner < 0 || r.preconditioner >= kPcCount) return fail(why, "unknown preconditioner model");
    if (r.gmres_restart <= 0) return fail(why, "the GMRES restart length must be positive");
    if (!std::isfinite(r.braess_sarazin_alpha) || !(r.braess_sarazin_alpha >= 0.25 && r.braess_sarazin_alpha <= 4.0))
        return fail(why, "the Braess-Sarazin alpha must lie in [0.25, 4]");
    if (!c.square) return fail(why, "automatic selection needs a square matrix");
    if (!kKrylovAvailable[r.krylov])
        return fail(why, std::string("Krylov model not implemented: ") + kKrylovNames[r.krylov]);
    if (!kPcAvailable[r.preconditioner])
        return fail(why, std::string("preconditioner model not implemented: ") + kPcNames[r.preconditioner]);

    std::memset(&plan, 0, sizeof(plan));
    plan.problem = problem;
    plan.automatic_krylov = r.krylov == kAuto;
    plan.automatic_preconditioner = r.preconditioner == pAuto;
    plan.null_space = r.null_space;
    const bool small = c.equations < 24;
    std::string reason;
    switch (problem) {
        case PressurePoisson:
        case Diffusion: {
            const bool spd_like = c.numerically_symmetric && c.diagonally_dominant && c.positive_diagonal;
            if (spd_like && c.strongly_directional_coupling && r.null_space != 1) {
                plan.krylov = kFGMRES;
                plan.preconditioner = small ? pJacobi : pNativeAMG;
                reason = "elliptic, directionally coupled: FGMRES with native AMG";
            } else if (spd_like && !c.large_diagonal_dynamic_range && !c.strongly_scaled) {
                plan.krylov = kCG;
                plan.preconditioner = small ? pJacobi : pNativeAMG;
                reason = "symmetric, diagonally dominant, moderately scaled: CG with an SPD preconditioner";
            } else {
                plan.krylov = kGMRES;
                plan.preconditioner = small ? pJacobi : pILU0;
                reason = "elliptic without an SPD signature: GMRES with a nonsymmetric-safe preconditioner";
            }
            break;
        }
        case Momentum:
        case ScalarTransport:
            plan.krylov = c.strongly_scaled ? kFGMRES : kBiCGStab;
            plan.preconditioner = small ? pJacobi : pILU0;
            reason = c.strongly_scaled ? "strongly scaled transport: FGMRES" : "transport: BiCGStab";
            break;
        case Coupled:
            if (!c.saddle_point) return fail(why, "coupled selection needs a saddle-point classification");
            plan.krylov = kFGMRES;
            plan.preconditioner = pCoupledBlockSchur;
            reason = "saddle point: FGMRES with a block Schur preconditioner";
            break;
        default:
            plan.krylov = kGMRES;
            plan.preconditioner = pJacobi;
            reason = "general operator: GMRES with Jacobi";
            break;
    }
    if (c.large_diagonal_dynamic_range) reason += "; large diagonal dynamic range";
    if (c.strongly_scaled) reason += "; strongly scaled coefficients";

    if (!plan.automatic_krylov) plan.krylov = r.krylov;
    if (!plan.automatic_preconditioner) plan.preconditioner = r.preconditioner;
    const int32_t pc = plan.preconditioner;
    const bool anisotropic_amg = pc == pAnisotropicBoomerAMG || pc == pAnisotropicSmoothedAggregationAMG ||
                                 pc == pDirectionalSemiCoarseningAMG || pc == pEnergyMinimizingAMG;
    // line and anisotropic AMG variants pair with a flexible outer method
    if (plan.automatic_krylov && (pc == pAnisotropicLineAMG || anisotropic_amg || pc == pAnisotropicLine)) {
        plan.krylov = kFGMRES;
        reason += "; line/anisotropic preconditioning: FGMRES";
    }
    // row or column equilibration is not a congruence: no CG
    const bool nonsymmetric_scaling = r.scaling >= 1 && r.scaling <= 3;
    if (plan.krylov == kCG && nonsymmetric_scaling) {
        if (!plan.automatic_krylov) return fail(why, "CG cannot use nonsymmetric scaling");
        plan.krylov = kFGMRES;
        reason += "; nonsymmetric scaling: FGMRES";
    }
    if (plan.null_space == 1 && plan.automatic_preconditioner) reason += "; constant null space projected";

    const bool cg_problem = problem == PressurePoisson || problem == Diffusion;
    const bool coupled = problem == Coupled;
    if (plan.krylov == kCG && (!cg_problem || !c.numerically_symmetric || !c.positive_diagonal))
        return fail(why, "CG needs a symmetric, positive-diagonal pressure or diffusion operator");
    if (plan.krylov == kCG && pc != pNone && pc != pJacobi && pc != pNativeAMG && pc != pSmoothedAggregationAMG)
        return fail(why, "CG needs an SPD-qualified preconditioner (none, Jacobi or native AMG)");
    if (pc == pAnisotropicLineAMG && (plan.krylov == kCG || coupled))
        return fail(why, "anisotropic line AMG needs a nonsymmetric scalar Krylov method");
    if ((pc == pNativeAMG || pc == pSmoothedAggregationAMG || anisotropic_amg) && !cg_problem)
        return fail(why, "native AMG is qualified for SPD elliptic problems only");
    if (anisotropic_amg && (!c.numerically_symmetric || !c.positive_diagonal))
        return fail(why, "anisotropic AMG needs a symmetric positive-diagonal operator");
    if ((pc == pBraessSarazin || pc == pVankaPressurePatch) && (!coupled || plan.krylov != kFGMRES))
        return fail(why, "Braess-Sarazin and Vanka are for coupled FGMRES only");
    if (pc == pNativeFieldSplit && !coupled) return fail(why, "field split needs a coupled problem");
    if ((pc == pCoupledBlockSchur || pc == pPCD || pc == pMGR) && !coupled)
        return fail(why, "block Schur, PCD and MGR need a coupled problem");
    if (plan.null_space == 1 && !cg_problem)
        return fail(why, "a constant null space is qualified for pressure and diffusion only");
    if (plan.null_space == 1 && plan.krylov != kCG && plan.krylov != kGMRES && plan.krylov != kFGMRES)
        return fail(why, "a constant null space needs CG, GMRES or FGMRES");
    std::snprintf(plan.reason, sizeof(plan.reason), "%s + %s: %s", kKrylovNames[plan.krylov], kPcNames[pc],
                  reason.c_str());
    return true;
}

}  // namespace cfdxg

namespace {
thread_local std::string g_plan_error;
}

extern "C" {

int cfdxg_measure_matrix_characteristics(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                                         int32_t saddle_point, double symmetry_tolerance,
                                         cfdxg_matrix_characteristics* out) {
    if (!out || !ro || n <= 0) {
        g_plan_error = "characteristics: empty or null matrix";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    if (!(symmetry_tolerance >= 0.0) || !std::isfinite(symmetry_tolerance)) {
        g_plan_error = "characteristics: the symmetry tolerance must be finite and non-negative";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    if (ro[0] != 0 || (ro[n] > 0 && (!co || !va))) {
        g_plan_error = "characteristics: invalid row offsets";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < n; ++i) {
        if (ro[i + 1] < ro[i]) {
            g_plan_error = "characteristics: row offsets decrease";
            return CFDXG_ERR_INVALID_ARGUMENT;
        }
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
            if (co[k] < 0 || co[k] >= n || (k > ro[i] && co[k] <= co[k - 1])) {
                g_plan_error = "characteristics: columns must increase strictly within [0, n)";
                return CFDXG_ERR_INVALID_ARGUMENT;
            }
    }
    cfdxg::measure_characteristics(n, ro, co, va, saddle_point != 0, symmetry_tolerance, *out);
    g_plan_error.clear();
    return CFDXG_OK;
}

int cfdxg_select_linear_solver(int32_t problem, const cfdxg_matrix_characteristics* c,
                               const cfdxg_plan_request* r, cfdxg_solver_plan* plan) {
    if (!c || !r || !plan) {
        g_plan_error = "plan: null argument";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    std::string why;
    if (!cfdxg::select_solver(problem, *c, *r, *plan, why)) {
        g_plan_error = why;
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    g_plan_error.clear();
    return CFDXG_OK;
}

int cfdxg_scale_matrix(int64_t n, const int64_t* ro, const int64_t* co, const double* va, int32_t scaling,
                       double zero_tolerance, double* row_scale, double* column_scale, double* scaled_values,
                       int64_t* zero_counts) {
    if (!ro || n <= 0 || !row_scale || !column_scale || !scaled_values || (ro[n] > 0 && (!co || !va))) {
        g_plan_error = "scaling: null argument";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    if (scaling < 0 || scaling > 4) {
        g_plan_error = "scaling: unknown scaling model";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    if (!(zero_tolerance >= 0.0) || !std::isfinite(zero_tolerance)) {
        g_plan_error = "scaling: the zero-row tolerance must be finite and non-negative";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
            if (co[k] < 0 || co[k] >= n) {
                g_plan_error = "scaling: column out of range";
                return CFDXG_ERR_INVALID_ARGUMENT;
            }
    int64_t zr = 0, zc = 0;
    cfdxg::scale_values(scaling, n, ro, co, va, zero_tolerance, row_scale, column_scale, scaled_values, zr, zc);
    if (zero_counts) {
        zero_counts[0] = zr;
        zero_counts[1] = zc;
    }
    g_plan_error.clear();
    return CFDXG_OK;
}

int cfdxg_diagnose_matrix(int64_t nr, int64_t nc, const int64_t* ro, const int64_t* co, const double* va,
                          double tol, int32_t topology, cfdxg_matrix_diagnostics* d) {
    if (!d || !ro || nr < 0 || nc < 0 || (nr > 0 && ro[nr] > 0 && (!co || !va))) {
        g_plan_error = "diagnosis: null argument";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    if (!(tol >= 0.0) || !std::isfinite(tol)) {
        g_plan_error = "diagnosis: the diagonal tolerance must be finite and non-negative";
        return CFDXG_ERR_INVALID_ARGUMENT;
    }
    const double inf = std::numeric_limits<double>::infinity();
    *d = cfdxg_matrix_diagnostics{};
    d->rows = nr;
    d->columns = nc;
    d->nnz = ro[nr];
    d->finite = 1;
    d->min_nonzero_abs_value = d->min_nonzero_row_sum = d->min_nonzero_column_sum = inf;
    d->min_nonzero_abs_diagonal = inf;
    d->diagonal_dynamic_range = d->row_sum_dynamic_range = d->column_sum_dynamic_range = 1.0;
    d->minimum_gershgorin_margin = inf;
    // SparseMatrix::is_consistent (sparse_matrix.h:256-275)
    bool consistent = ro[0] == 0;
    for (int64_t i = 0; i < nr && consistent; ++i) {
        if (ro[i + 1] < ro[i]) consistent = false;
        for (int64_t k = ro[i]; k < ro[i + 1] && consistent; ++k)
            if (co[k] < 0 || co[k] >= nc || !std::isfinite(va[k]) || (k > ro[i] && co[k] <= co[k - 1]))
                consistent = false;
    }
    d->structurally_consistent = consistent;
    if (!consistent) {
        d->finite = 0;
        g_plan_error.clear();
        return CFDXG_OK;
    }
    std::vector<double> row_sum(static_cast<size_t>(nr), 0.0), col_sum(static_cast<size_t>(nc), 0.0);
    std::vector<char> row_off(static_cast<size_t>(nr), 0), col_off(static_cast<size_t>(nc), 0);
    for (int64_t i = 0; i < nr; ++i) {
        if (ro[i] == ro[i + 1]) ++d->empty_rows;
        bool present = false;
        double diagonal = 0.0;
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
            const int64_t j = co[k];
            const double m = std::fabs(va[k]);
            d->max_abs_value = cfdxg::ref_max(d->max_abs_value, m);
            if (m > 0.0) d->min_nonzero_abs_value = cfdxg::ref_min(d->min_nonzero_abs_value, m);
            row_sum[i] += m;
            col_sum[j] += m;
            if (j == i) {
                present = true;
                diagonal += va[k];
            } else if (m > 0.0) {
                row_off[i] = 1;
                col_off[j] = 1;
            }
        }
        if (!present && i < nc) ++d->missing_diagonal;
        const double dabs = std::fabs(diagonal);
        if (dabs > 0.0) {
            d->max_abs_diagonal = cfdxg::ref_max(d->max_abs_diagonal, dabs);
            d->min_nonzero_abs_diagonal = cfdxg::ref_min(d->min_nonzero_abs_diagonal, dabs);
        }
        // against the running max |a| over the rows so far, as the reference's loop has it
        if (i < nc && dabs <= tol * cfdxg::ref_max(1.0, d->max_abs_value)) ++d->near_zero_diagonal;
        if (i < nc) {
            double off = 0.0;
            for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
                if (co[k] != i) off += std::fabs(va[k]);
            d->minimum_gershgorin_margin = cfdxg::ref_min(d->minimum_gershgorin_margin, dabs - off);
        }
    }
    for (int64_t j = 0; j < nc; ++j)
        if (col_sum[j] == 0.0) ++d->empty_columns;
    for (int64_t i = 0; i < std::min(nr, nc); ++i)
        if (!row_off[i] && !col_off[i]) ++d->isolated_dofs;
    for (const double v : row_sum)
        if (v > 0.0) {
            d->max_row_sum = cfdxg::ref_max(d->max_row_sum, v);
            d->min_nonzero_row_sum = cfdxg::ref_min(d->min_nonzero_row_sum, v);
        }
    for (const double v : col_sum)
        if (v > 0.0) {
            d->max_column_sum = cfdxg::ref_max(d->max_column_sum, v);
            d->min_nonzero_column_sum = cfdxg::ref_min(d->min_nonzero_column_sum, v);
        }
    if (d->min_nonzero_abs_diagonal < inf) d->diagonal_dynamic_range = d->max_abs_diagonal / d->min_nonzero_abs_diagonal;
    if (d->min_nonzero_row_sum < inf) d->row_sum_dynamic_range = d->max_row_sum / d->min_nonzero_row_sum;
    if (d->min_nonzero_column_sum < inf)
        d->column_sum_dynamic_range = d->max_column_sum / d->min_nonzero_column_sum;
    if (nr != nc) d->minimum_gershgorin_margin = std::numeric_limits<double>::quiet_NaN();
    if (topology) {
        // components of the bipartite graph (row nodes, then column nodes), nonzero entries as edges
        std::vector<int64_t> parent(static_cast<size_t>(nr + nc));
        for (int64_t v = 0; v < nr + nc; ++v) parent[v] = v;
        auto find = [&](int64_t v) {
            while (parent[v] != v) v = parent[v] = parent[parent[v]];
            return v;
        };
        int64_t components = nr + nc;
        for (int64_t i = 0; i < nr; ++i)
            for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
                if (std::fabs(va[k]) == 0.0) continue;
                const int64_t a = find(i), b = find(nr + co[k]);
                if (a != b) {
                    parent[a] = b;
                    --components;
                }
            }
        d->connected_components = components;
    }
    g_plan_error.clear();
    return CFDXG_OK;
}

const char* cfdxg_plan_last_error(void) { return g_plan_error.c_str(); }

}  // extern "C"
